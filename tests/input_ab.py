"""The reference's input-format A/B checks, restated for this scorer.

Each case encodes the same content two ways: frame A in the format under
test, frame B as linear float RGB (or float 4:4:4) whose samples come from
the reference's independent FP64 model of the conversions,
tests/input/input_reference.h, written from the standards rather than from
the shader code. The pair must then score like (B, B):

    MaxNormDelta(Compute(A, B), Compute(B, B)) <= tolerance

with the reference's bounds (tests/input/input_format_test_support.h:61-71):
2e-4, 4e-4 for PQ and HLG. Cases, content and formats follow
tests/input/input_format_test.cc:207-433 and
tests/input/input_format_chroma_test.cc:104-430.

The FP64 values are computed once by tests/golden/make_input_ab.py through
oracle/_ref/libvqm_ref.so (input_reference.h compiled from the reference
checkout) and kept in tests/golden/input_ab.npz, so the checks run where
the reference checkout is absent; the CPU tests compare the fixture with the
live library whenever it is built.
"""

from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

from tests import helpers
from vqm_b200 import ss2

SIDE = 32                 # vqm::test::kSide
ROUNDING = 2e-4           # kRounding
PQ_CURVE = 4e-4           # kPqCurve
HLG_CURVE = 4e-4          # kHlgCurve
FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "input_ab.npz")

T, M, Pr = ss2.TransferCharacteristics, ss2.MatrixCoefficients, ss2.ColorPrimaries
L, CF = ss2.ChromaLocation, ss2.ChromaFilter

# input_format_test.cc:283-302: every transfer swept over half its domain
# (`upper` = the top half); the log and PQ curves get both halves.
TRANSFER_CASES = [
    (T.Bt709, False), (T.Bt601, False), (T.Bt2020_10, False), (T.Bt2020_12, False),
    (T.St240M, False), (T.Bt470M, False), (T.Bt470Bg, False), (T.Srgb, False),
    (T.Log100, True), (T.Log316, True), (T.Iec61966_2_4, True), (T.Bt1361, True),
    (T.St428, False), (T.Linear, False), (T.St2084, True), (T.St2084, False),
    (T.AribB67, True), (T.AribB67, False),
]
HLG_CHROMATIC = (0.4, 0.55, 0.7)  # input_format_test.cc:350-352
# input_format_test.cc:370-384: (matrix, primaries, chromaticity-derived).
MATRIX_CASES = [
    (M.Bt709, Pr.Bt709, False), (M.Bt470Bg, Pr.Bt709, False), (M.St170M, Pr.Bt709, False),
    (M.St240M, Pr.Bt709, False), (M.Fcc, Pr.Bt709, False), (M.YCgCo, Pr.Bt709, False),
    (M.Bt2020Ncl, Pr.Bt2020, False), (M.Bt2020Ncl, Pr.Bt470Bg, False),
    (M.ChromaticityDerivedNcl, Pr.Bt2020, True), (M.ChromaticityDerivedNcl, Pr.Bt470Bg, True),
    (M.ChromaticityDerivedNcl, Pr.Ebu3213E, True),
]
PRIMARIES_CASES = [Pr.Bt470M, Pr.Bt470Bg, Pr.St170M, Pr.St240M, Pr.Film, Pr.Bt2020, Pr.St428,
                   Pr.St431_2, Pr.St432_1, Pr.Ebu3213E]  # input_format_test.cc:420-425
# input_format_chroma_test.cc:146-161: (sub_w, sub_h, filter, siting).
SUBSAMPLING_CASES = [
    (1, 1, CF.Bilinear, L.Left), (1, 1, CF.Bicubic, L.Left), (1, 1, CF.Lanczos, L.Left),
    (1, 0, CF.Bilinear, L.Left), (2, 0, CF.Bilinear, L.Left), (1, 1, CF.Bilinear, L.Center),
    (1, 1, CF.Bilinear, L.TopLeft), (1, 1, CF.Bilinear, L.Top),
    (1, 1, CF.Bilinear, L.BottomLeft), (1, 1, CF.Bilinear, L.Bottom),
    (1, 1, CF.Bicubic, L.Bottom),
]
CL_YUV = (0.5, 0.1, -0.2)                      # input_format_chroma_test.cc:261
CL_CASES = [(M.Bt2020Cl, Pr.Bt2020), (M.ChromaticityDerivedCl, Pr.Bt709),
            (M.ChromaticityDerivedCl, Pr.Bt470Bg)]
ICTCP = (0.5, 0.15, -0.12)                     # input_format_chroma_test.cc:305
ICTCP_CASES = [(T.St2084, 100.0), (T.AribB67, 10.0)]


def ramp_index() -> np.ndarray:
    """x + y per pixel (the ramp depends on nothing else)."""
    return np.add.outer(np.arange(SIDE), np.arange(SIDE))


def ramp(k):
    """Ramp(x, y) of input_format_test.cc:55-59 for k = x + y."""
    return 0.02 + 0.96 * (np.asarray(k, dtype=np.float64) / (2.0 * (SIDE - 1)))


def transfer_sample(upper: bool, k):
    v = ramp(k)
    return 0.5 + 0.5 * v if upper else 0.5 * v


def matrix_plane(k):
    t = ramp(k)
    return np.stack([0.1 + 0.8 * t, 0.25 - 0.4 * t, -0.25 + 0.5 * t], axis=-1)


def primaries_sample(k):
    t = ramp(k)
    return np.stack([0.1 + 0.8 * t, 0.9 - 0.8 * t, 0.05 + 0.5 * t], axis=-1)


def subsampled_content(sw: int, sh: int):
    """SubsampledContent (input_format_chroma_test.cc:14-37): an 8-bit-exact
    luma ramp and a sharp chroma edge at the chroma planes' centre."""
    y = np.tile((np.arange(SIDE, dtype=np.float32) / np.float32(SIDE - 1)), (SIDE, 1))
    cw, ch = SIDE >> sw, SIDE >> sh
    u = np.where(np.arange(cw)[None, :] < cw // 2, 0.2, 0.8) * np.ones((ch, 1))
    v = np.where(np.arange(ch)[:, None] < ch // 2, 0.7, 0.3) * np.ones((1, cw))
    return [y, u.astype(np.float32), v.astype(np.float32), None]


# ---------------------------------------------------------------------------
# The reference's FP64 model, through oracle/_ref/libvqm_ref.so
# ---------------------------------------------------------------------------


class Reference:
    """input_reference.h's functions (oracle/input_ref_shim.cc)."""

    def __init__(self, lib: ctypes.CDLL):
        d, p, i, u = ctypes.c_double, ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32
        lib.vqmin_decode_transfer.restype = d
        lib.vqmin_decode_transfer.argtypes = [i, d]
        lib.vqmin_hlg_to_linear.argtypes = [p, d, d, d, d, p]
        lib.vqmin_ncl_to_rgb.argtypes = [i, p]
        lib.vqmin_ncl_to_rgb_from_primaries.argtypes = [i, p]
        lib.vqmin_gamut.argtypes = [i, i, p]
        lib.vqmin_yuv_constants_from_primaries.argtypes = [i, p, p]
        lib.vqmin_cl_to_rgb.argtypes = [d, d, p, p]
        lib.vqmin_ictcp_to_lms.argtypes = [i, p]
        lib.vqmin_lms_to_rgb.argtypes = [p]
        lib.vqmin_axis_taps.restype = i
        lib.vqmin_axis_taps.argtypes = [i, u, d, d, u, p, p, i]
        lib.vqmin_chroma_shift.restype = d
        lib.vqmin_chroma_shift.argtypes = [i, i, u]
        self.lib = lib

    def _mat(self, fn, *args) -> np.ndarray:
        out = np.zeros(9)
        fn(*args, out.ctypes.data)
        return out.reshape(3, 3)

    def decode(self, transfer, v: float) -> float:
        return self.lib.vqmin_decode_transfer(int(transfer), float(v))

    def hlg(self, v, kr, kg, kb, scale) -> np.ndarray:
        src, out = np.asarray(v, dtype=np.float64), np.zeros(3)
        self.lib.vqmin_hlg_to_linear(src.ctypes.data, kr, kg, kb, scale, out.ctypes.data)
        return out

    def ncl(self, matrix):
        return self._mat(self.lib.vqmin_ncl_to_rgb, int(matrix))

    def ncl_from_primaries(self, primaries):
        return self._mat(self.lib.vqmin_ncl_to_rgb_from_primaries, int(primaries))

    def gamut(self, src, dst):
        return self._mat(self.lib.vqmin_gamut, int(src), int(dst))

    def kr_kb(self, primaries):
        kr, kb = ctypes.c_double(), ctypes.c_double()
        self.lib.vqmin_yuv_constants_from_primaries(int(primaries), ctypes.byref(kr),
                                                    ctypes.byref(kb))
        return kr.value, kb.value

    def cl_to_rgb(self, kr, kb, yuv) -> np.ndarray:
        src, out = np.asarray(yuv, dtype=np.float64), np.zeros(3)
        self.lib.vqmin_cl_to_rgb(kr, kb, src.ctypes.data, out.ctypes.data)
        return out

    def ictcp_to_lms(self, transfer):
        return self._mat(self.lib.vqmin_ictcp_to_lms, int(transfer))

    def lms_to_rgb(self):
        return self._mat(self.lib.vqmin_lms_to_rgb)

    def axis_taps(self, filt, out_pos, scale, shift, dim):
        idx, w = np.zeros(16, dtype=np.uint32), np.zeros(16)
        n = self.lib.vqmin_axis_taps(int(filt), out_pos, scale, shift, dim, idx.ctypes.data,
                                     w.ctypes.data, 16)
        return list(zip(idx[:n].tolist(), w[:n].tolist()))

    def chroma_shift(self, location, horizontal, subsample) -> float:
        return self.lib.vqmin_chroma_shift(int(location), int(horizontal), subsample)


def _mul(m: np.ndarray, v) -> np.ndarray:
    """ref::Mul(Mat3, Vec3): (m0 v0 + m1 v1) + m2 v2 per row, in double."""
    v = [float(x) for x in v]
    return np.array([(m[r, 0] * v[0] + m[r, 1] * v[1]) + m[r, 2] * v[2] for r in range(3)])


def reference_values(ref: Reference) -> dict:
    """Every FP64 value the cases take from input_reference.h, rounded to
    float as the reference tests store them (std::vector<float>)."""
    out = {}
    ks = np.arange(2 * SIDE - 1)
    for transfer, upper in TRANSFER_CASES:
        vals = []
        for k in ks:
            v = float(transfer_sample(upper, k))
            if transfer == T.AribB67:
                vals.append(ref.hlg([v, v, v], 0.2126, 0.7152, 0.0722, 10.0)[0])
            else:
                vals.append(ref.decode(transfer, v))
        out[f"transfer_{transfer}_{int(upper)}"] = np.array(vals, dtype=np.float32)
    out["transfer_hlg_chromatic"] = ref.hlg(HLG_CHROMATIC, 0.2126, 0.7152, 0.0722,
                                            10.0).astype(np.float32)
    for matrix, prim, derived in MATRIX_CASES:
        ncl = ref.ncl_from_primaries(prim) if derived else ref.ncl(matrix)
        to_target = ref.gamut(prim, Pr.Bt709)
        out[f"matrix_{matrix}_{prim}"] = np.array(
            [_mul(to_target, _mul(ncl, p)) for p in matrix_plane(ks)], dtype=np.float32)
    for prim in PRIMARIES_CASES:
        to_target = ref.gamut(prim, Pr.Bt709)
        out[f"primaries_{prim}"] = np.array([_mul(to_target, p) for p in primaries_sample(ks)],
                                            dtype=np.float32)
    for sw, sh, filt, loc in SUBSAMPLING_CASES:
        src = subsampled_content(sw, sh)
        cw, ch = SIDE >> sw, SIDE >> sh
        sx, sy = ref.chroma_shift(loc, True, sw), ref.chroma_shift(loc, False, sh)
        up = np.zeros((2, SIDE, SIDE), dtype=np.float32)
        for y in range(SIDE):
            ty = ref.axis_taps(filt, y, float(1 << sh), sy, ch)
            for x in range(SIDE):
                tx = ref.axis_taps(filt, x, float(1 << sw), sx, cw)
                for c in (0, 1):
                    acc = 0.0
                    for iy, wy in ty:
                        for ix, wx in tx:
                            acc += wx * wy * float(src[1 + c][iy, ix])
                    up[c, y, x] = acc
        out[f"subsampling_{sw}{sh}_{filt}_{loc}"] = up
    for matrix, prim in CL_CASES:
        kr, kb = (0.2627, 0.0593) if matrix == M.Bt2020Cl else ref.kr_kb(prim)
        rgb = ref.cl_to_rgb(kr, kb, CL_YUV)
        out[f"cl_{matrix}_{prim}"] = _mul(ref.gamut(prim, Pr.Bt709), rgb).astype(np.float32)
    for transfer, scale in ICTCP_CASES:
        lms = _mul(ref.ictcp_to_lms(transfer), ICTCP)
        if transfer == T.AribB67:
            decoded = ref.hlg(lms, 0.2627, 0.6780, 0.0593, scale)
        else:
            decoded = np.array([ref.decode(transfer, x) for x in lms])
        rgb = _mul(ref.gamut(Pr.Bt2020, Pr.Bt709), _mul(ref.lms_to_rgb(), decoded))
        out[f"ictcp_{transfer}"] = rgb.astype(np.float32)
    return out


def live_reference() -> Reference | None:
    from oracle import binding as ob
    lib = ob.ref()
    if lib is None or not hasattr(lib, "vqmin_decode_transfer"):
        return None
    return Reference(lib)


def load_fixture() -> dict:
    with np.load(FIXTURE) as f:
        return {k: f[k] for k in f.files}


# ---------------------------------------------------------------------------
# The cases
# ---------------------------------------------------------------------------


@dataclass
class Case:
    name: str
    a: ss2.Image
    b: ss2.Image
    tolerance: float
    background: float = 0.5
    chroma_filter: int = 0


def _pack(fmt, values, w=SIDE, h=SIDE):
    return helpers.pack_planes(fmt, w, h, [None if v is None else np.asarray(v, np.float32)
                                           for v in values])


def _uniform(rgb, alpha=1.0):
    return [np.full((SIDE, SIDE), float(np.float32(c)), dtype=np.float32) for c in rgb] + [
        np.full((SIDE, SIDE), alpha, dtype=np.float32)]


def _per_pixel(table: np.ndarray):
    """Planes from a table indexed by x + y ([63] or [63, 3])."""
    k = ramp_index()
    t = np.asarray(table, dtype=np.float32)
    if t.ndim == 1:
        return [t[k], t[k], t[k], None]
    return [t[k, 0], t[k, 1], t[k, 2], None]


def linear_rgb():
    """LinearRgbFormat (input_format_test_support.h:90-97)."""
    return ss2.ImageFormat(type=ss2.PixelType.Float, transfer=T.Linear, primaries=Pr.Bt709)


def yuv_format(sw, sh, loc):
    """YuvFormat (input_format_chroma_test.cc:76-89)."""
    return ss2.ImageFormat(type=ss2.PixelType.Float, family=ss2.ColorFamily.Yuv,
                           matrix=M.Bt709, transfer=T.Linear, primaries=Pr.Bt709,
                           subsample_w=sw, subsample_h=sh, chroma_location=loc)


def ladder(grid: int):
    """Ladder(grid, 0) (input_format_test.cc:12-31)."""
    x = np.arange(SIDE)[None, :].repeat(SIDE, 0)
    y = np.arange(SIDE)[:, None].repeat(SIDE, 1)
    r = (x * 7) % (grid + 1)
    g = (y * 13) % (grid + 1)
    b = (x * 11 + y * 5) % (grid + 1)
    return [(c / float(grid)).astype(np.float32) for c in (r, g, b)] + [None]


def cases(values: dict) -> list[Case]:
    out = []
    base = helpers.pinned_format()  # PinnedFormat(None): float sRGB
    # Datatypes, depth and range (input_format_test.cc:207-279).
    half = base.copy(type=ss2.PixelType.Half)
    out.append(Case("half vs float", _pack(half, ladder(1024)), _pack(base, ladder(1024)),
                    ROUNDING))
    word = base.copy(type=ss2.PixelType.Word, depth=16)
    out.append(Case("word16 vs float", _pack(word, ladder(65535)), _pack(base, ladder(65535)),
                    ROUNDING))
    byte = base.copy(type=ss2.PixelType.Byte)
    out.append(Case("byte vs float", _pack(byte, ladder(255)), _pack(base, ladder(255)),
                    ROUNDING))
    word10 = base.copy(type=ss2.PixelType.Word, depth=10)
    out.append(Case("word10 vs float", _pack(word10, ladder(1023)), _pack(base, ladder(1023)),
                    ROUNDING))
    limited = byte.copy(range=ss2.PixelRange.Limited)
    # Not a rounding bound: the two decimations differ by up to half a
    # limited-range code step (input_format_test.cc:262-278).
    out.append(Case("limited vs full", _pack(limited, ladder(255)), _pack(byte, ladder(255)),
                    1e-2))
    # Transfer functions (input_format_test.cc:281-347).
    k = ramp_index()
    for transfer, upper in TRANSFER_CASES:
        fmt = base.copy(transfer=transfer)
        v = transfer_sample(upper, k)
        a = _pack(fmt, [v, v, v, None])
        b = _pack(linear_rgb(), _per_pixel(values[f"transfer_{transfer}_{int(upper)}"]))
        tol = PQ_CURVE if transfer == T.St2084 else HLG_CURVE if transfer == T.AribB67 \
            else ROUNDING
        out.append(Case(f"transfer {transfer} {'upper' if upper else 'lower'}", a, b, tol))
    fmt = base.copy(transfer=T.AribB67)
    out.append(Case("transfer HLG chromatic", _pack(fmt, _uniform(HLG_CHROMATIC)[:3] + [None]),
                    _pack(linear_rgb(), _uniform(values["transfer_hlg_chromatic"])[:3] + [None]),
                    HLG_CURVE))
    # Matrix coefficients (input_format_test.cc:361-409).
    for matrix, prim, _ in MATRIX_CASES:
        fmt = ss2.ImageFormat(type=ss2.PixelType.Float, family=ss2.ColorFamily.Yuv,
                              matrix=matrix, transfer=T.Linear, primaries=prim)
        plane = matrix_plane(k)
        a = _pack(fmt, [plane[..., 0], plane[..., 1], plane[..., 2], None])
        b = _pack(linear_rgb(), _per_pixel(values[f"matrix_{matrix}_{prim}"]))
        out.append(Case(f"matrix {matrix} primaries {prim}", a, b, ROUNDING))
    # Primaries (input_format_test.cc:413-433).
    for prim in PRIMARIES_CASES:
        fmt = linear_rgb().copy(primaries=prim)
        s = primaries_sample(k)
        a = _pack(fmt, [s[..., 0], s[..., 1], s[..., 2], None])
        b = _pack(linear_rgb(), _per_pixel(values[f"primaries_{prim}"]))
        out.append(Case(f"primaries {prim}", a, b, ROUNDING))
    # The absolute code mapping of full-range byte chroma
    # (input_format_chroma_test.cc:104-142): codes Y 128, U 128, V 255.
    fmt = yuv_format(0, 0, L.Left).copy(type=ss2.PixelType.Byte)
    data = np.zeros(ss2.required_bytes(fmt, SIDE, SIDE), dtype=np.uint8)
    for p, code in enumerate((128, 128, 255)):
        off = ss2.plane_layout(fmt, SIDE, SIDE)[p][0]
        data[off:off + SIDE * SIDE] = code
    coded = ss2.Image(SIDE, SIDE, fmt, data)
    ref_img = _pack(yuv_format(0, 0, L.Left),
                    _uniform((128.0 / 255.0, 0.0, 127.0 / 255.0))[:3] + [None])
    out.append(Case("full-range byte chroma", coded, ref_img, ROUNDING))
    # Subsampling, chroma filters and sitings (input_format_chroma_test.cc:144-186).
    for sw, sh, filt, loc in SUBSAMPLING_CASES:
        a = _pack(yuv_format(sw, sh, loc), subsampled_content(sw, sh))
        up = values[f"subsampling_{sw}{sh}_{filt}_{loc}"]
        b = _pack(yuv_format(0, 0, loc), [subsampled_content(0, 0)[0], up[0], up[1], None])
        out.append(Case(f"subsampling {sw}x{sh} filter {filt} siting {loc}", a, b, ROUNDING,
                        chroma_filter=int(filt)))
    # Constant luminance and ICtCp (input_format_chroma_test.cc:258-339).
    for matrix, prim in CL_CASES:
        fmt = ss2.ImageFormat(type=ss2.PixelType.Float, family=ss2.ColorFamily.Yuv,
                              matrix=matrix, transfer=T.Bt709, primaries=prim)
        out.append(Case(f"CL matrix {matrix} primaries {prim}",
                        _pack(fmt, _uniform(CL_YUV)[:3] + [None]),
                        _pack(linear_rgb(), _uniform(values[f"cl_{matrix}_{prim}"])[:3] + [None]),
                        ROUNDING))
    for transfer, _ in ICTCP_CASES:
        fmt = ss2.ImageFormat(type=ss2.PixelType.Float, family=ss2.ColorFamily.Yuv,
                              matrix=M.Bt2100ICtCp, transfer=transfer, primaries=Pr.Bt2020)
        out.append(Case(f"ictcp transfer {transfer}", _pack(fmt, _uniform(ICTCP)[:3] + [None]),
                        _pack(linear_rgb(), _uniform(values[f"ictcp_{transfer}"])[:3] + [None]),
                        HLG_CURVE if transfer == T.AribB67 else ROUNDING))
    # Alpha types: straight alpha A over colour S equals premultiplied S*A
    # (input_format_chroma_test.cc:343-378), on two backgrounds.
    x = np.arange(SIDE)[None, :].repeat(SIDE, 0)
    y = np.arange(SIDE)[:, None].repeat(SIDE, 1)
    alpha = ((x + 3 * y) % 7) / 6.0
    s = [x / (SIDE - 1), y / (SIDE - 1), ((x * 7 + y * 11) % 64) / 63.0]
    straight = [c.astype(np.float32) for c in s] + [alpha.astype(np.float32)]
    premul = [(c * alpha).astype(np.float32) for c in s] + [alpha.astype(np.float32)]
    a = _pack(helpers.pinned_format(alpha=ss2.AlphaType.Straight), straight)
    b = _pack(helpers.pinned_format(alpha=ss2.AlphaType.Premultiplied), premul)
    for bg in (0.1, 0.9):
        out.append(Case(f"alpha types background {bg}", a, b, ROUNDING, background=bg))
    return out


def max_norm_delta(a: np.ndarray, b: np.ndarray) -> float:
    """MaxNormDelta (input_format_test_support.h:106-127): the largest
    absolute difference over every feature of every scale."""
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    if a.shape != b.shape:
        return 1e9
    return float(np.max(np.abs(a - b)))
