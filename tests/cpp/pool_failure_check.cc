// Ssimulacra2Pool's failure path in include/vqm_cuda.hpp, without a device:
// the C ABI calls the pool makes on its workers are replaced, at link time
// (ld --wrap), by fakes that fail on the host where the test says so.
//
// Checked, after the reference's src/pool.cc:44-109:
//   1. a submission that fails in the middle of a list: every chunk already
//      submitted is finished before the error propagates, and the pool stays
//      usable;
//   2. a finish that fails: the other chunks in flight are still finished,
//      the first error propagates, and the pool stays usable;
//   3. a failure whose drain fails too: the workers are released and every
//      later call throws std::logic_error("pool cannot be reused after a
//      failed drain").
// Exit status 0 when every check holds.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#include "vqm_cuda.hpp"

namespace v = vqm::cuda;

namespace {

struct FakeBatch {
    std::uint64_t next_token = 1;
    std::set<std::uint64_t> in_flight;
};

int g_batches = 0;               // live fake batches
int g_submits = 0;               // submissions so far (all batches)
int g_fail_submit_at = -1;       // fail the submission with this ordinal
std::set<int> g_fail_finish;     // fail the finishes with these ordinals
int g_finishes = 0;              // finishes so far
std::string g_error;

int Fail(int status, const char* what) {
    g_error = what;
    return status;
}

}  // namespace

extern "C" {

int __wrap_vqm_cu_ss2_batch_create(const vqm_cu_ss2_batch_config*, vqm_cu_ss2_batch** out) {
    *out = reinterpret_cast<vqm_cu_ss2_batch*>(new FakeBatch());
    ++g_batches;
    return VQM_CU_OK;
}

int __wrap_vqm_cu_ss2_batch_destroy(vqm_cu_ss2_batch* b) {
    delete reinterpret_cast<FakeBatch*>(b);
    --g_batches;
    return VQM_CU_OK;
}

int __wrap_vqm_cu_ss2_batch_submit_borrowed(vqm_cu_ss2_batch* b, uint32_t, const vqm_cu_image*,
                                            const vqm_cu_image*, float, uint64_t* token) {
    auto* f = reinterpret_cast<FakeBatch*>(b);
    if (!f->in_flight.empty()) return Fail(VQM_CU_LOGIC_ERROR, "fake: a batch is in flight");
    if (g_submits++ == g_fail_submit_at)
        return Fail(VQM_CU_INVALID_ARGUMENT, "fake: invalid image in the list");
    *token = f->next_token++;
    f->in_flight.insert(*token);
    return VQM_CU_OK;
}

int __wrap_vqm_cu_ss2_batch_finish(vqm_cu_ss2_batch* b, uint64_t token, double* norms,
                                   uint32_t* scales, double*) {
    auto* f = reinterpret_cast<FakeBatch*>(b);
    if (!f->in_flight.erase(token)) return Fail(VQM_CU_INVALID_ARGUMENT, "fake: stale token");
    if (g_fail_finish.count(g_finishes++))
        return Fail(VQM_CU_RUNTIME_ERROR, "fake: the device reported an error");
    if (norms) std::memset(norms, 0, sizeof(double) * VQM_CU_SS2_MAX_NORMS);
    if (scales) *scales = 1;
    return VQM_CU_OK;
}

const char* __wrap_vqm_cu_last_error(void) { return g_error.c_str(); }

}  // extern "C"

namespace {

int failures = 0;

void Expect(bool ok, const char* what) {
    if (!ok) {
        std::fprintf(stderr, "FAIL: %s\n", what);
        ++failures;
    }
}

// n pairs of one 8x8 image (ImagePair holds references: `img` outlives them).
std::vector<v::ImagePair> Pairs(const v::Image& img, std::size_t n) {
    return std::vector<v::ImagePair>(n, v::ImagePair{img, img});
}

v::Image Blank() {
    v::ImageFormat fmt;
    fmt.type = v::PixelType::Byte;
    v::Image img;
    img.size = {8, 8};
    img.format = fmt;
    img.data.assign(v::RequiredBytes(fmt, img.size), 0);
    return img;
}

void Reset() {
    g_submits = 0;
    g_finishes = 0;
    g_fail_submit_at = -1;
    g_fail_finish.clear();
}

}  // namespace

int main() {
    const v::Image blank = Blank();
    const auto pairs = Pairs(blank, 10);  // chunks of 2 over 3 workers: 5 submissions
    {
        v::Ssimulacra2Pool pool(v::Ssimulacra2Config{{8, 8}}, 3, 2);
        Reset();
        Expect(pool.ComputeMany(pairs).size() == 10, "a clean list returns every result");
        Expect(g_submits == 5 && g_finishes == 5, "a clean list finishes every chunk");

        // 1. The fourth submission fails: the three chunks before it are
        // finished, then the submission's error propagates.
        Reset();
        g_fail_submit_at = 3;
        bool threw = false;
        try {
            (void)pool.ComputeMany(pairs);
        } catch (const std::invalid_argument& e) {
            threw = std::string(e.what()) == "fake: invalid image in the list";
        }
        Expect(threw, "a failed submission propagates its own error");
        Expect(g_finishes == 3, "every chunk submitted before the failure is finished");
        Reset();
        Expect(pool.ComputeMany(pairs).size() == 10 && pool.Workers() == 3,
               "the pool is usable after a drained failure");

        // 2. The second finish fails: the chunks still in flight are
        // finished, the first error propagates, the pool stays usable.
        Reset();
        g_fail_finish = {1};
        threw = false;
        try {
            (void)pool.ComputeMany(pairs);
        } catch (const std::runtime_error& e) {
            threw = std::string(e.what()) == "fake: the device reported an error";
        }
        Expect(threw, "a failed finish propagates its error");
        Expect(g_finishes == g_submits, "every submitted chunk was finished");
        Reset();
        Expect(pool.ComputeMany(pairs).size() == 10, "usable after a failed finish");

        // 3. A submission fails and a finish of the drain fails too: the
        // pool releases its workers and refuses every later call.
        Reset();
        g_fail_submit_at = 3;
        g_fail_finish = {1};
        threw = false;
        try {
            (void)pool.ComputeMany(pairs);
        } catch (const std::invalid_argument&) {
            threw = true;  // the error that interrupted the list, not the drain's
        }
        Expect(threw, "the interrupting error propagates, not the drain's");
        Expect(g_batches == 0 && pool.Workers() == 0, "a failed drain releases the workers");
        std::string message;
        try {
            (void)pool.ComputeMany(pairs);
        } catch (const std::logic_error& e) {
            message = e.what();
        }
        Expect(message == "pool cannot be reused after a failed drain",
               "a poisoned pool refuses further use");
    }
    Expect(g_batches == 0, "no fake batch leaks");
    if (failures == 0) std::printf("pool failure checks passed\n");
    return failures == 0 ? 0 : 1;
}
