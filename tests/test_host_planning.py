"""Host-side planning (csrc/qb_common.cuh, csrc/qb_tc.cuh, csrc/qb_tc2.cuh), checked on the
CPU: the record geometries, the tie order, the tensor-core shard plan, and the 16-bit pair
form's eligibility, unit and constants.

The kernel reads each accumulator as a 16-bit value v(u) = D(u) + s*X(u) - Dmin - lo_s
(F = D~ + 2^23 - Dlow_s in fp32, low half of the bit pattern) and adds one packed constant:
per chunk c = (u4, u5, u6) for tile t, giving D(u) - Dmin, and per position k = (u1, u2, u3),
half u0 and column half u7 for the partner tile, giving D(u) + s*gamma(u) - Dmin, all modulo
2^16.  The harness (tests/host_planning_harness.cpp) exports the library's own table builder
and planning functions; this test emulates the kernel's arithmetic with them."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "evo-quantum-qubolib_b200", "csrc")
CUDA_INC = "/usr/local/cuda/include"


class Tc2Tab(ctypes.Structure):
    _fields_ = [("gx", ctypes.c_float * 3), ("k0s", ctypes.c_float * 2), ("dmin", ctypes.c_float),
                ("corr_t", (ctypes.c_uint32 * 8) * 2), ("corr_p", ((ctypes.c_uint32 * 8) * 2) * 2)]


@pytest.fixture(scope="module")
def harness(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None or not os.path.isdir(CUDA_INC):
        pytest.skip("g++ or the CUDA headers are not available")
    out = str(tmp_path_factory.mktemp("planning") / "host_planning.so")
    subprocess.run([gxx, "-std=c++17", "-O1", "-fPIC", "-shared", "-I", CSRC, "-I", CUDA_INC,
                    os.path.join(HERE, "host_planning_harness.cpp"), "-o", out], check=True)
    L = ctypes.CDLL(out)
    dp, fp = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_float)
    L.h_tc2_u16_eligible.argtypes = [ctypes.c_int, dp, fp]
    L.h_tc2_u16_quantized.argtypes = [ctypes.c_int, dp, ctypes.c_double, dp, fp, dp]
    L.h_tc2_u16_tables.argtypes = [fp, ctypes.c_float, ctypes.POINTER(Tc2Tab)]
    L.h_tc_plan.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                            ctypes.POINTER(ctypes.c_uint64), dp, ctypes.POINTER(ctypes.c_int)]
    L.h_record_states.argtypes = [ctypes.c_int] * 9 + [ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                                                      ctypes.POINTER(ctypes.c_uint64)]
    L.h_grayrank64.argtypes = [ctypes.c_uint64]
    L.h_grayrank64.restype = ctypes.c_uint64
    L.h_tie_key.argtypes = [ctypes.c_int] * 5 + [ctypes.c_uint64]
    L.h_tie_key.restype = ctypes.c_uint64
    assert L.h_tc2_tab_size() == ctypes.sizeof(Tc2Tab)
    return L


def _tables(L, gamma, dmin):
    g = np.asarray(gamma, dtype=np.float32)
    t = Tc2Tab()
    L.h_tc2_u16_tables(g.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), float(dmin), ctypes.byref(t))
    return t


def _half(word, d):
    return (int(word) >> (16 * d)) & 0xFFFF


@pytest.mark.parametrize("seed", range(6))
def test_corrections_recover_both_tiles(harness, seed):
    rng = np.random.default_rng(seed)
    gamma = rng.integers(-2000, 2001, 8)
    if seed == 0:
        gamma[[4, 5, 6]] = [2000, -2000, 0]  # extreme and zero chunk couplings
    dmin = float(rng.integers(-40000, 1000))
    t = _tables(harness, gamma, dmin)
    u = np.arange(256)
    bit = lambda b: (u >> b) & 1  # noqa: E731
    X = sum(int(gamma[b]) * bit(b) for b in (4, 5, 6))
    gam = sum(int(gamma[b]) * bit(b) for b in range(8))
    c, k, d, hh = (u >> 4) & 7, (u >> 1) & 7, u & 1, u >> 7
    assert [int(v) for v in t.gx] == [int(gamma[b]) for b in (4, 5, 6)] and t.dmin == dmin
    margin = int(np.abs(gamma).sum())
    for neg, s in ((0, 1), (1, -1)):
        lo = sum(min(0, s * int(gamma[b])) for b in (4, 5, 6))
        assert t.k0s[neg] == 2.0 ** 23 - (dmin + lo)
        for trial in range(4):
            # accumulator values D(u) whose partner values D + s*gamma(u) are values too
            D = dmin + margin + rng.integers(0, 30000, 256)
            v = D + s * X - dmin - lo
            assert v.min() >= 0 and v.max() < 1 << 16  # the 16-bit read is exact
            for j in range(256):
                ct = _half(t.corr_t[neg][c[j]], d[j])
                assert _half(t.corr_t[neg][c[j]], 0) == _half(t.corr_t[neg][c[j]], 1)
                assert (int(v[j]) + ct) & 0xFFFF == D[j] - dmin
                cp = _half(t.corr_p[neg][hh[j]][k[j]], d[j])
                assert (int(v[j]) + cp) & 0xFFFF == D[j] + s * gam[j] - dmin


def _upper(rng, n, scale):
    W = np.triu(rng.standard_normal((n, n)) * scale)
    return W


@pytest.mark.parametrize("n,scale,seed", [(24, 1.0, 0), (30, 37.5, 1), (36, 0.01, 2), (36, 1e4, 3)])
def test_rounded_unit_is_the_largest_power_of_two_within_limits(harness, n, scale, seed):
    rng = np.random.default_rng(seed)
    W = _upper(rng, n, scale)
    abs_sum = float(np.abs(W).sum())
    sg, dm, ep = ctypes.c_double(), ctypes.c_float(), ctypes.c_double()
    dp = ctypes.POINTER(ctypes.c_double)
    ok = harness.h_tc2_u16_quantized(n, W.ctypes.data_as(dp), abs_sum, ctypes.byref(sg), ctypes.byref(dm),
                                     ctypes.byref(ep))
    assert ok == 1
    sigma = sg.value
    assert sigma > 0 and np.log2(sigma) == int(np.log2(sigma))  # a power of two
    # the kernel's limits, restated from the W entries the 16-bit form reads
    rows = [W[n - 9 - i, n - 8:] for i in range(7)]
    rowmax = max(max(r[r > 0].sum(), -r[r < 0].sum()) for r in rows)
    vals = [W[n - 9 - i, n - 1 - j] for i in range(7) for j in range(8)]
    for j in range(8):
        a = n - 1 - j
        vals += [W[a, a]] + [W[a, n - 1 - j2] for j2 in range(j)] + [W[t, a] for t in range(n - 15)]
    vals = np.array(vals)
    lo, hi = vals[vals < 0].sum(), vals[vals > 0].sum()
    gA = sum(abs(W[n - 16, n - 1 - b]) for b in (4, 5, 6))

    def fits(sg):
        return sg * rowmax <= 2047 and sg * (hi - lo + gA) + 40 <= 65535

    assert fits(sigma) and not fits(2 * sigma) and sigma * (hi - lo) >= 1024
    assert dm.value == np.floor(sigma * lo) - 12
    assert ep.value == pytest.approx(10 / sigma + abs_sum * 2.0 ** -16, rel=1e-15)


def test_rounded_form_refuses_a_coarse_or_empty_span(harness):
    dp = ctypes.POINTER(ctypes.c_double)
    sg, dm, ep = ctypes.c_double(), ctypes.c_float(), ctypes.c_double()
    n = 26
    Z = np.zeros((n, n))  # no couplings touch the u variables: zero span
    assert harness.h_tc2_u16_quantized(n, Z.ctypes.data_as(dp), 0.0, ctypes.byref(sg), ctypes.byref(dm),
                                       ctypes.byref(ep)) == 0
    assert harness.h_tc2_u16_quantized(19, Z.ctypes.data_as(dp), 0.0, ctypes.byref(sg), ctypes.byref(dm),
                                       ctypes.byref(ep)) == 0  # below 20 variables


def test_exact_eligibility_needs_room_for_the_chunk_couplings(harness):
    """Integer W whose value span fits 16 bits but not with the chunk couplings added."""
    n = 24
    fp = ctypes.c_float()
    dp = ctypes.POINTER(ctypes.c_double)
    W = np.zeros((n, n))
    W[n - 16, n - 1 - 4] = 100.0  # a chunk coupling of the pair variable
    assert harness.h_tc2_u16_eligible(n, W.ctypes.data_as(dp), ctypes.byref(fp)) == 1
    # the value span counts the coupling (100) once; the chunk offset adds |gamma_4| = 100
    W[n - 1, n - 1] = 65535.0 - 200.0  # span + offset = 2^16 - 1: still exact in 16 bits
    assert harness.h_tc2_u16_eligible(n, W.ctypes.data_as(dp), ctypes.byref(fp)) == 1
    assert fp.value == 0.0  # Dmin: no negative couplings
    W[n - 1, n - 1] = 65535.0 - 199.0  # span + offset = 2^16: refused, though the span fits
    assert harness.h_tc2_u16_eligible(n, W.ctypes.data_as(dp), ctypes.byref(fp)) == 0


def _plan(L, n, is_int, abs_sum, idx, cnt, gl=0):
    u = (ctypes.c_uint64 * 5)()
    f = (ctypes.c_double * 2)()
    i = (ctypes.c_int * 3)()
    L.h_tc_plan(n, int(is_int), float(abs_sum), idx, cnt, gl, u, f, i)
    return {"tile_begin": u[0], "tile_end": u[1], "rec_begin": u[2], "rec_count": u[3], "states": u[4],
            "scale": f[0], "eps": f[1], "nt": i[0], "gl": i[1], "exact": i[2]}


@pytest.mark.parametrize("n", [20, 21, 24, 29, 33, 36, 40])
def test_shard_plans_partition_the_tiles_on_record_blocks(harness, n):
    """Shards of any count (more shards than record blocks included) cover every Gray tile
    and every record exactly once, in order, each boundary on a record block; the exact flag
    and the digit scale follow the stated rules."""
    for gl in (0, 5, n - 15, n - 14):  # n - 14 is out of range: the default applies
        for cnt in (1, 2, 3, 7, 8, 64):
            plans = [_plan(harness, n, True, 1000.0, s, cnt, gl) for s in range(cnt)]
            g = plans[0]["gl"]
            assert g == (gl if 5 <= gl <= n - 15 else max(5, n - 33))
            tile, rec = 0, 0
            for p in plans:
                assert p["tile_begin"] == tile and p["rec_begin"] == rec
                assert p["tile_begin"] % (1 << g) == 0 and p["tile_end"] % (1 << g) == 0
                assert p["rec_count"] == ((p["tile_end"] - p["tile_begin"]) >> g) * 8
                assert p["states"] == (p["tile_end"] - p["tile_begin"]) << 15
                tile, rec = p["tile_end"], p["rec_begin"] + p["rec_count"]
            assert tile == 1 << (n - 15) and rec == 8 << (n - 15 - g)
            assert sum(p["states"] for p in plans) == 1 << n
    # exact integer digits up to sum|Q| = 2^22; beyond, and for float Q, a power-of-two scale
    # with scale * sum|Q| <= 2^14 < 2 * scale * sum|Q| and a positive error bound
    for is_int, s in ((True, 2.0 ** 22), (True, 2.0 ** 22 + 1), (False, 3.0), (False, 12345.678), (False, 1e-3)):
        p = _plan(harness, n, is_int, s, 0, 1)
        exact = is_int and s <= 2.0 ** 22
        assert p["exact"] == int(exact)
        if exact:
            assert p["scale"] == 1.0 and p["eps"] == 0.0
        else:
            assert p["scale"] * s <= 2.0 ** 14 < 2 * p["scale"] * s and p["eps"] > 0


GEOM_GRAY, GEOM_TC, GEOM_BLOCK = 1, 2, 3


def _covered(L, geom, count):
    """Every state of every record 0..count-1, as one array (records share one free mask)."""
    base, free = ctypes.c_uint64(), ctypes.c_uint64()
    bases, masks = [], set()
    for r in range(count):
        L.h_record_states(*geom, r, ctypes.byref(base), ctypes.byref(free))
        bases.append(base.value)
        masks.add(free.value)
    assert len(masks) == 1
    m = masks.pop()
    pos = [i for i in range(64) if (m >> i) & 1]
    sub = np.zeros(1 << len(pos), dtype=np.uint64)
    for i, p in enumerate(pos):
        sub |= ((np.arange(1 << len(pos), dtype=np.uint64) >> np.uint64(i)) & np.uint64(1)) << np.uint64(p)
    b = np.array(bases, dtype=np.uint64)
    assert not np.any(b & np.uint64(m))  # the base leaves the free bits clear
    return (b[:, None] | sub[None, :]).ravel()


def _gray_geoms(n):
    for b in sorted({13, max(13, n - 16), n - 7}):
        a = n - b
        if not (7 <= a <= 24):
            continue
        cb = b - 13
        for sbits in sorted({5, a, min(a, max(5, n - 34))}):
            for ubits in sorted({max(7, sbits), a}):
                if ubits < sbits or ubits > a:
                    continue
                gub = ubits - sbits
                count = 1 << (a - ubits + cb + gub + 3)
                yield (GEOM_GRAY, n, a, b, sbits, cb, gub, 0, 0), count


@pytest.mark.parametrize("n", [20, 21, 22])
def test_records_partition_the_states(harness, n):
    """Each geometry's records, expanded to states, cover every one of the 2^n states exactly
    once (pass 2 re-walks exactly the states of the selected records)."""
    geoms = list(_gray_geoms(n))
    nt = n - 15
    for gl in sorted({5, nt}):
        geoms.append(((GEOM_TC, n, 0, 0, 0, 0, 0, gl, 0), 8 << (nt - gl)))
    geoms.append(((GEOM_BLOCK, n, 0, 0, 0, 0, 0, 0, min(n, 16)), 1 << (n - min(n, 16))))
    assert len(geoms) >= 4
    for geom, count in geoms:
        states = _covered(harness, geom, count)
        assert states.size == 1 << n, geom
        assert int(states.max()) < 1 << n
        hits = np.bincount(states.astype(np.int64), minlength=1 << n)
        assert hits.min() == 1 and hits.max() == 1, geom


def test_grayrank_inverts_the_gray_code(harness):
    rng = np.random.default_rng(4)
    for i in [0, 1, 2, 3, (1 << 63) - 1, (1 << 64) - 1] + [int(v) for v in rng.integers(0, 1 << 63, 200)]:
        g = i ^ (i >> 1)
        assert harness.h_grayrank64(g) == i


TIE_QBF, TIE_QBF1 = 0, 1


@pytest.mark.parametrize("n,k,A", [(20, 0, 0), (24, 0, 4), (30, 0, 10), (36, 0, 16), (30, 3, 7), (36, 5, 11),
                                   (40, 0, 20), (44, 2, 22)])
def test_qbf_tie_order_is_the_oracles(harness, n, k, A):
    """Sorting states by the library's tie key gives the order of the reference's prefix loop
    (QBF: inverse-Gray rank of the prefix, then the suffix; under Parallel the task bits
    first), as the oracle states it."""
    import oracle
    B = n - k - A
    rng = np.random.default_rng(n * 100 + k)
    xs = [int(v) for v in rng.integers(0, 1 << n, 300, dtype=np.uint64)]
    xs += [x for x in (0, (1 << n) - 1, 1 << (n - 1), 1 << B, (1 << B) - 1) if x < 1 << n]
    mine = sorted(xs, key=lambda x: harness.h_tie_key(TIE_QBF, n, k, A, B, x))
    if k == 0:
        ref = sorted(xs, key=lambda x: oracle.qbf_key(x, n, A))
    else:
        ref = sorted(xs, key=lambda x: oracle.parallel_key(x, n, k, A))
    assert mine == ref


@pytest.mark.parametrize("n,k", [(19, 0), (24, 0), (33, 0), (44, 0), (30, 2)])
def test_qb_f1_tie_order_is_the_oracles(harness, n, k):
    """QB_F1's answer order: task bits, then the thread of the reference kernel that owns the
    18-bit suffix column, then the Gray step of the prefix (src/qubo_lib/solvers/qbf1.py:195-249)."""
    import oracle
    A = n - k - 18
    rng = np.random.default_rng(n)
    xs = [int(v) for v in rng.integers(0, 1 << n, 300, dtype=np.uint64)] + [0, (1 << n) - 1]
    mine = sorted(xs, key=lambda x: harness.h_tie_key(TIE_QBF1, n, k, A, 18, x))
    mask = (1 << 18) - 1
    ref = sorted(xs, key=lambda x: (x >> (n - k) if k else 0, oracle.qbf1_tid(x & mask),
                                    oracle.grayrank((x >> 18) & ((1 << A) - 1))))
    assert mine == ref


EXACT_MAX_FREE = 40  # free bits of one record that the exact re-walk takes (csrc/qb_exact.cuh)


@pytest.mark.parametrize("n", list(range(20, 63)))
def test_tensor_core_records_stay_within_the_exact_rewalk(harness, n):
    """Every record of the tensor-core form (2^gl tiles x 128 rows x 256 columns of a block:
    gl + 12 free bits) must fit the exact re-walk, for the default record size and for every
    override the plan accepts, up to the library's largest n."""
    nt = n - 15
    p = _plan(harness, n, True, 1000.0, 0, 1)
    assert p["gl"] + 12 <= EXACT_MAX_FREE, p
    for gl in range(5, nt + 2):
        q = _plan(harness, n, True, 1000.0, 0, 1, gl)
        assert q["gl"] + 12 <= EXACT_MAX_FREE, (gl, q)
        assert q["gl"] == gl or q["gl"] == p["gl"]  # an accepted override, else the default
