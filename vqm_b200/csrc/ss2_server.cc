// Serving loop: continuous batching of single-pair requests over a few batch
// scorers (vqm_cu_ss2_batch_*), each with its own stream and device memory.
//
// Requests queue in arrival order. The dispatcher thread takes a free worker
// whenever one exists and fills a batch from the head of the queue while its
// pair count stays within max_batch_pairs and the device memory the worker
// will hold for it, plus what every other worker holds, stays within the
// budget (memory counted as allocated, growth included: the workers' own
// report, vqm_cu_ss2_batch_device_bytes[_after]). When the head request does
// not fit, idle workers' memory is freed (vqm_cu_ss2_batch_trim); if it still
// does not fit, it waits for running batches to finish. The batch scorer
// copies host inputs (waiting for the copies, so the dispatcher is the only
// thread feeding PCIe) and launches its two kernels. The completion thread finishes batches in the
// order they were submitted (blocking on each batch's completion event),
// publishes the results and returns the worker. So requests that arrive while
// batches run are admitted as soon as a worker frees, and up to `workers`
// batches overlap on the device (one's copies beside another's kernels).
//
// A request's result does not depend on the batch it lands in: every pair
// is prepared, blurred and reduced by its own CTAs, and its partials are
// summed in a fixed order per pair.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda_runtime_api.h>

#include "../../include/vqm_cu_ss2.h"
#include "ss2_host.h"
#include "ss2_kernels.h"
#include "ss2_layout.h"

namespace vqm_b200 {
namespace {

using Clock = std::chrono::steady_clock;

size_t Align(size_t v, size_t a) { return (v + a - 1) / a * a; }

// Device bytes one pair adds to a batch: its pyramid, tile partials, segment
// sums, result block, table records and (for host images) the staged copy
// of its inputs, as the batch scorer lays them out, with room to spare for
// alignment: an upper bound of what a batch of this pair alone allocates.
size_t PairDeviceBytes(const vqm_cu_image& o, const vqm_cu_image& d, int variant) {
    int tw = 0, th = 0;
    BlurTileShape(variant, &tw, &th);
    const ScalePlan plan = PlanScales(o.width, o.height);
    size_t floats = 0, tiles = 0, segs = 0;
    for (int l = 0; l < plan.count; ++l)
        for (int c = 0; c < 3; ++c) {
            if (!(plan.mask[l] & (1u << c))) continue;
            floats += PlaneFloats(plan.w[l], plan.h[l]);
            tiles += static_cast<size_t>((plan.w[l] + tw - 1) / tw) * ((plan.h[l] + th - 1) / th);
            ++segs;
        }
    size_t bytes = Align(2 * floats, 64) * sizeof(float) + tiles * 6 * sizeof(double) +
                   segs * (6 * sizeof(double) + sizeof(DevSegment) + sizeof(uint32_t)) +
                   kResultDoubles * sizeof(double) + sizeof(DevPair) + 4096;
    for (const vqm_cu_image* img : {&o, &d})
        if (img->memory == VQM_CU_MEMORY_HOST)
            bytes += Align(RequiredBytes(img->format, img->width, img->height), 256);
    return bytes;
}

struct Request {
    vqm_cu_image o{}, d{};
    float background = 0.5f;
    size_t bytes = 0;
    Clock::time_point submitted, completed;
    bool done = false;
    int status = VQM_CU_OK;
    std::string error;
    double norms[108] = {};
    uint32_t scales = 0;
    double score = 0.0;
};

class Server {
public:
    explicit Server(const vqm_cu_ss2_server_config& cfg) {
        budget_ = cfg.memory_budget ? cfg.memory_budget : (40ull << 30);
        const uint32_t workers = cfg.workers ? cfg.workers : 2;
        max_pairs_ = cfg.max_batch_pairs ? cfg.max_batch_pairs : 64;
        if (workers > 64) throw std::invalid_argument("server: at most 64 workers");
        if (cfg.chroma_filter > 2) throw std::invalid_argument("invalid chroma filter");
        if (cfg.variant > static_cast<uint32_t>(BlurTileCount()))
            throw std::invalid_argument("cuda: no such blur variant");
        variant_ = cfg.variant ? static_cast<int>(cfg.variant) - 1 : kDefaultBlurVariant;
        BlurTaps(cfg.blur);  // rejects an unknown blur mode
        ClampToFreeMemory(cfg.device);
        stats_.budget_bytes = budget_;
        for (uint32_t i = 0; i < workers; ++i) {
            vqm_cu_ss2_batch_config bc{};
            bc.max_pairs = max_pairs_;
            bc.chroma_filter = cfg.chroma_filter;
            bc.device = cfg.device;
            bc.variant = cfg.variant;
            bc.blur = cfg.blur;
            vqm_cu_ss2_batch* b = nullptr;
            if (vqm_cu_ss2_batch_create(&bc, &b) != VQM_CU_OK) {
                const std::string msg = vqm_cu_last_error();
                for (auto& w : workers_) vqm_cu_ss2_batch_destroy(w.batch);
                throw std::runtime_error(msg);
            }
            workers_.push_back(Worker{b});
            free_.push_back(i);
        }
        dispatcher_ = std::thread([this] { Dispatch(); });
        completer_ = std::thread([this] { Complete(); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lock(mu_);
            stop_ = true;
        }
        work_cv_.notify_all();
        inflight_cv_.notify_all();
        dispatcher_.join();
        completer_.join();
        for (auto& w : workers_) vqm_cu_ss2_batch_destroy(w.batch);
    }

    uint64_t Submit(const vqm_cu_image& o, const vqm_cu_image& d, float background) {
        if (o.width != d.width || o.height != d.height)
            throw std::invalid_argument("distorted: image size does not match the original");
        ValidateFormat(o.format, o.width, o.height, "original");
        ValidateFormat(d.format, d.width, d.height, "distorted");
        for (const vqm_cu_image* img : {&o, &d})
            if (img->memory != VQM_CU_MEMORY_HOST && img->memory != VQM_CU_MEMORY_DEVICE)
                throw std::invalid_argument("server: invalid memory kind");
        auto r = std::make_unique<Request>();
        r->o = o;
        r->d = d;
        r->background = background;
        r->bytes = PairDeviceBytes(o, d, variant_);
        if (r->bytes > budget_)
            throw std::invalid_argument(
                "server: a " + std::to_string(o.width) + "x" + std::to_string(o.height) +
                " pair needs " + std::to_string(r->bytes) + " device bytes; the budget is " +
                std::to_string(budget_));
        uint64_t ticket;
        {
            std::lock_guard<std::mutex> lock(mu_);
            if (stop_) throw std::logic_error("server: shutting down");
            ticket = ++next_ticket_;
            r->submitted = Clock::now();
            requests_.emplace(ticket, std::move(r));
            queue_.push_back(ticket);
            ++stats_.submitted;
            stats_.queued = queue_.size();
        }
        work_cv_.notify_one();
        return ticket;
    }

    // VQM_CU_OK, VQM_CU_TIMEOUT, or the failed request's status (message in
    // `error`).
    int Wait(uint64_t ticket, int32_t timeout_ms, double* norms, uint32_t* scales, double* score,
             double* latency_ms, std::string& error) {
        std::unique_lock<std::mutex> lock(mu_);
        auto it = requests_.find(ticket);
        if (it == requests_.end()) throw std::invalid_argument("server: no request with that ticket");
        Request* r = it->second.get();
        const auto ready = [r] { return r->done; };
        if (timeout_ms < 0) {
            done_cv_.wait(lock, ready);
        } else if (!done_cv_.wait_for(lock, std::chrono::milliseconds(timeout_ms), ready)) {
            return VQM_CU_TIMEOUT;
        }
        if (norms) std::memcpy(norms, r->norms, sizeof(r->norms));
        if (scales) *scales = r->scales;
        if (score) *score = r->score;
        if (latency_ms)
            *latency_ms = std::chrono::duration<double, std::milli>(r->completed - r->submitted).count();
        const int status = r->status;
        error = r->error;
        requests_.erase(it);
        return status;
    }

    vqm_cu_ss2_server_stats Stats() {
        std::lock_guard<std::mutex> lock(mu_);
        return stats_;
    }

private:
    struct Worker {
        vqm_cu_ss2_batch* batch = nullptr;
        std::vector<uint64_t> tickets;
        uint64_t token = 0;
        size_t bytes = 0;  // what the batch's requests need
        size_t held = 0;   // device memory the batch scorer holds
    };

    // The budget in force: memory_budget, or the device's free memory less
    // 256 MiB when that is smaller.
    void ClampToFreeMemory(int32_t device) {
        int current = 0;
        if (cudaGetDevice(&current) != cudaSuccess) {
            cudaGetLastError();
            throw std::runtime_error("cuda: no device");
        }
        const int want = ResolveDeviceOrdinal(device);
        size_t free_bytes = 0, total = 0;
        const bool ok = cudaSetDevice(want) == cudaSuccess &&
                        cudaMemGetInfo(&free_bytes, &total) == cudaSuccess;
        cudaSetDevice(current);
        if (!ok) {
            cudaGetLastError();
            throw std::runtime_error("cuda: cannot read the device's free memory");
        }
        const size_t margin = size_t(256) << 20;
        if (free_bytes > margin) budget_ = std::min(budget_, free_bytes - margin);
    }

    // With the lock held: whether worker `w`, holding what it will hold once
    // `os`/`ds` are submitted to it (its own count; nothing is allocated),
    // fits the budget beside `others`. A submission the worker cannot count
    // is let through: its submit fails and reports why.
    bool Fits(Worker& w, const std::vector<vqm_cu_image>& os,
              const std::vector<vqm_cu_image>& ds, size_t others) {
        uint64_t after = 0;
        if (vqm_cu_ss2_batch_device_bytes_after(w.batch, static_cast<uint32_t>(os.size()),
                                                os.data(), ds.data(), &after) != VQM_CU_OK)
            return true;
        return others <= budget_ && after <= budget_ - others;
    }

    void SetHeld(Worker& w, size_t held) {
        stats_.device_bytes = stats_.device_bytes - w.held + held;
        stats_.peak_device_bytes = std::max(stats_.peak_device_bytes, stats_.device_bytes);
        w.held = held;
    }

    // With the lock held: frees the memory of the idle workers (`wi`, the
    // one being filled, included) that hold any. Returns whether it freed any.
    bool TrimIdle() {
        bool freed = false;
        for (int i : free_)
            if (workers_[i].held && vqm_cu_ss2_batch_trim(workers_[i].batch) == VQM_CU_OK) {
                SetHeld(workers_[i], 0);
                ++stats_.trims;
                freed = true;
            }
        return freed;
    }

    void Dispatch() {
        std::unique_lock<std::mutex> lock(mu_);
        for (;;) {
            work_cv_.wait(lock, [this] { return stop_ || (!queue_.empty() && !free_.empty()); });
            if (queue_.empty()) {
                if (stop_) break;
                continue;
            }
            if (free_.empty()) continue;
            const int wi = free_.front();
            Worker& w = workers_[wi];
            w.tickets.clear();
            w.bytes = 0;
            std::vector<vqm_cu_image> os, ds;
            float background = 0.5f;
            const size_t others = stats_.device_bytes - w.held;
            // Take requests while their estimate fits, then shrink the batch
            // until the worker's own count of the memory it will hold fits.
            while (!queue_.empty() && w.tickets.size() < max_pairs_) {
                Request* r = requests_.at(queue_.front()).get();
                // One background per batch: a request with another one starts
                // the next batch.
                if (!w.tickets.empty() && r->background != background) break;
                if (!w.tickets.empty() && (others > budget_ ||
                                           w.bytes + r->bytes > budget_ - others))
                    break;
                background = r->background;
                w.bytes += r->bytes;
                w.tickets.push_back(queue_.front());
                os.push_back(r->o);
                ds.push_back(r->d);
                queue_.pop_front();
            }
            while (!w.tickets.empty() && !Fits(w, os, ds, others)) {
                queue_.push_front(w.tickets.back());
                w.bytes -= requests_.at(w.tickets.back())->bytes;
                w.tickets.pop_back();
                os.pop_back();
                ds.pop_back();
            }
            if (w.tickets.empty()) {
                // The head request does not fit beside what the workers hold:
                // free the idle workers' memory and try again, or wait for a
                // running batch to finish (and become idle) first.
                if (TrimIdle()) continue;
                if (!inflight_.empty()) {
                    // The completer finishes in-flight batches whether or
                    // not the server is stopping, so this wait ends.
                    const uint64_t seen = completions_;
                    work_cv_.wait(lock, [&] { return completions_ != seen; });
                    continue;
                }
                // Everything is idle and freed, and still no fit: the pair is
                // larger than the budget by the workers' exact count.
                Request* r = requests_.at(queue_.front()).get();
                r->status = VQM_CU_INVALID_ARGUMENT;
                r->error = "server: the pair needs more device memory than the budget";
                r->completed = Clock::now();
                r->done = true;
                ++stats_.failed;
                queue_.pop_front();
                stats_.queued = queue_.size();
                done_cv_.notify_all();
                continue;
            }
            free_.pop_front();
            stats_.queued = queue_.size();
            stats_.bytes_in_flight += w.bytes;
            stats_.peak_bytes = std::max(stats_.peak_bytes, stats_.bytes_in_flight);
            stats_.largest_batch = std::max<uint64_t>(stats_.largest_batch, w.tickets.size());
            lock.unlock();
            uint64_t token = 0;
            const int rc = vqm_cu_ss2_batch_submit(w.batch, static_cast<uint32_t>(os.size()),
                                                   os.data(), ds.data(), background, &token);
            const std::string msg = rc == VQM_CU_OK ? std::string() : vqm_cu_last_error();
            uint64_t held = 0;
            if (vqm_cu_ss2_batch_device_bytes(w.batch, &held) != VQM_CU_OK) held = w.held;
            lock.lock();
            SetHeld(w, static_cast<size_t>(held));
            if (rc != VQM_CU_OK) {
                Fail(w, rc, msg);
                free_.push_back(wi);
                inflight_cv_.notify_one();  // the completer may be waiting to stop
                continue;
            }
            w.token = token;
            ++stats_.batches;
            inflight_.push_back(wi);
            inflight_cv_.notify_one();
        }
        inflight_cv_.notify_one();
    }

    void Complete() {
        std::unique_lock<std::mutex> lock(mu_);
        std::vector<double> norms, scores;
        std::vector<uint32_t> scales;
        for (;;) {
            // Stop once nothing is queued or in flight and the dispatcher
            // has been told to stop (it drains the queue first).
            inflight_cv_.wait(lock, [this] {
                return !inflight_.empty() || (stop_ && queue_.empty() && dispatch_idle());
            });
            if (inflight_.empty()) break;
            const int wi = inflight_.front();
            Worker& w = workers_[wi];
            const size_t n = w.tickets.size();
            lock.unlock();
            norms.assign(n * 108, 0.0);
            scores.assign(n, 0.0);
            scales.assign(n, 0);
            const int rc = vqm_cu_ss2_batch_finish(w.batch, w.token, norms.data(), scales.data(),
                                                   scores.data());
            const std::string msg = rc == VQM_CU_OK ? std::string() : vqm_cu_last_error();
            const auto now = Clock::now();
            lock.lock();
            inflight_.pop_front();
            if (rc != VQM_CU_OK) {
                Fail(w, rc, msg);
            } else {
                for (size_t i = 0; i < n; ++i) {
                    Request* r = requests_.at(w.tickets[i]).get();
                    std::memcpy(r->norms, norms.data() + i * 108, sizeof(r->norms));
                    r->scales = scales[i];
                    r->score = scores[i];
                    r->completed = now;
                    r->done = true;
                }
                stats_.completed += n;
                stats_.bytes_in_flight -= w.bytes;
            }
            free_.push_back(wi);
            ++completions_;
            done_cv_.notify_all();
            work_cv_.notify_one();
        }
    }

    // With the lock held: every worker is free or in flight, none is being
    // filled by the dispatcher.
    bool dispatch_idle() const { return free_.size() + inflight_.size() == workers_.size(); }

    void Fail(Worker& w, int rc, const std::string& msg) {
        const auto now = Clock::now();
        for (uint64_t t : w.tickets) {
            Request* r = requests_.at(t).get();
            r->status = rc;
            r->error = msg;
            r->completed = now;
            r->done = true;
        }
        stats_.failed += w.tickets.size();
        stats_.bytes_in_flight -= w.bytes;
        done_cv_.notify_all();
    }

    size_t budget_ = 0;
    uint64_t completions_ = 0;  // batches finished, for a dispatcher waiting on one
    uint32_t max_pairs_ = 64;
    int variant_ = 0;
    std::vector<Worker> workers_;
    std::mutex mu_;
    std::condition_variable work_cv_, inflight_cv_, done_cv_;
    std::deque<uint64_t> queue_;
    std::deque<int> free_, inflight_;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests_;
    uint64_t next_ticket_ = 0;
    bool stop_ = false;
    vqm_cu_ss2_server_stats stats_{};
    std::thread dispatcher_, completer_;
};

template <class F>
int GuardServer(F&& f) {
    try {
        f();
        SetLastErrorMessage("");
        return VQM_CU_OK;
    } catch (const std::invalid_argument& e) {
        SetLastErrorMessage(e.what());
        return VQM_CU_INVALID_ARGUMENT;
    } catch (const std::logic_error& e) {
        SetLastErrorMessage(e.what());
        return VQM_CU_LOGIC_ERROR;
    } catch (const std::overflow_error& e) {
        SetLastErrorMessage(e.what());
        return VQM_CU_OVERFLOW_ERROR;
    } catch (const std::exception& e) {
        SetLastErrorMessage(e.what());
        return VQM_CU_RUNTIME_ERROR;
    }
}

}  // namespace
}  // namespace vqm_b200

struct vqm_cu_ss2_server {
    vqm_b200::Server impl;
    explicit vqm_cu_ss2_server(const vqm_cu_ss2_server_config& c) : impl(c) {}
};

extern "C" {

int vqm_cu_ss2_server_create(const vqm_cu_ss2_server_config* config, vqm_cu_ss2_server** server) {
    return vqm_b200::GuardServer([&] {
        if (!config || !server) throw std::invalid_argument("config and server must not be null");
        *server = new vqm_cu_ss2_server(*config);
    });
}

int vqm_cu_ss2_server_destroy(vqm_cu_ss2_server* server) {
    return vqm_b200::GuardServer([&] { delete server; });
}

int vqm_cu_ss2_server_submit(vqm_cu_ss2_server* server, const vqm_cu_image* original,
                             const vqm_cu_image* distorted, float background, uint64_t* ticket) {
    return vqm_b200::GuardServer([&] {
        if (!server || !original || !distorted || !ticket)
            throw std::invalid_argument("server, images and ticket must not be null");
        *ticket = server->impl.Submit(*original, *distorted, background);
    });
}

int vqm_cu_ss2_server_wait(vqm_cu_ss2_server* server, uint64_t ticket, int32_t timeout_ms,
                           double* norms108, uint32_t* scales, double* score, double* latency_ms) {
    int status = VQM_CU_OK;
    std::string error;
    const int rc = vqm_b200::GuardServer([&] {
        if (!server) throw std::invalid_argument("server must not be null");
        status = server->impl.Wait(ticket, timeout_ms, norms108, scales, score, latency_ms, error);
    });
    if (rc != VQM_CU_OK) return rc;
    if (status == VQM_CU_TIMEOUT) vqm_b200::SetLastErrorMessage("server: the wait timed out");
    else if (status != VQM_CU_OK) vqm_b200::SetLastErrorMessage(error.c_str());
    return status;
}

int vqm_cu_ss2_server_get_stats(vqm_cu_ss2_server* server, vqm_cu_ss2_server_stats* stats) {
    return vqm_b200::GuardServer([&] {
        if (!server || !stats) throw std::invalid_argument("server and stats must not be null");
        *stats = server->impl.Stats();
    });
}

}  // extern "C"
