"""The algebra the GPU kernels rely on, checked in float64 on the CPU.

1. The scaled 5-operation form (uniform gap qualities with ins == del):
   with c = mi*gapm the sweep keeps M~ = mi*M, I^ = I, D^ = D of the
   reference's DP (src/core/pairhmm/intra/pairhmm_impl.cpp:245-290, row 0
   D = init, column 0 zero, likelihood = sum of the last row's M + I) via
       M~ = (e*c) * ((mm/c)*M~_d + I^_d + D^_d)
       I^ = ii*I^_u + M~_u
       D^ = dd*D^_l + M~_l
   over 32R rows, rows past the read's end L being pass-through rows
   (emission 0; the first takes ii = mi, the next ones ii = 1).  The
   likelihood is (sum of the last row's I^)/mi when that row is a pass-through
   row, else sum(M~_L)/mi + sum(I^_L).
2. The bound behind the multi-pass early rejection: every alignment emits
   read row r from M or I at some column and the rest of a path multiplies by
   factors <= 1, so the likelihood is at most sum_j (M + I)[r][j] for every
   row r, per-row gap qualities included.
3. The chain sweeps' sum row (float32, one rounding per operation): D + M of
   a last row with emission 1 and dd = 1 at a separator column is bitwise the
   running sum of the pass-through value over the haplotype's columns.

The priors here are plain float64 formulas (ph2pr[q] = 10^(-q/10), mm = 1 -
ph2pr[ins] - ph2pr[del]); both forms use the same ones, so the comparison is
of the recurrences, not of the reference's tables.
"""
import numpy as np
import pytest


def ph2pr(q):
    return 10.0 ** (-np.asarray(q, dtype=np.float64) / 10.0)


def priors(read_q, ins, dele, gcp):
    e = ph2pr(read_q)
    return dict(match=1.0 - e, mismatch=e / 3.0, mi=ph2pr(ins), md=ph2pr(dele),
                ii=ph2pr(gcp), dd=ph2pr(gcp), gapm=1.0 - ph2pr(gcp),
                mm=1.0 - (ph2pr(ins) + ph2pr(dele)))


def emissions(read, hap, p):
    eq = read[:, None] == hap[None, :]
    return np.where(eq, p["match"][:, None], p["mismatch"][:, None])


def reference_dp(read, hap, p, init):
    """The reference form; returns (M, I, D) of rows 1..L, columns 0..H."""
    L, H = len(read), len(hap)
    E = emissions(read, hap, p)
    M = np.zeros((L + 1, H + 1)); I = np.zeros_like(M); D = np.zeros_like(M)
    D[0, 1:] = init
    for i in range(1, L + 1):
        r = i - 1
        M[i, 1:] = E[r] * (p["mm"][r] * M[i - 1, :-1] +
                           p["gapm"][r] * (I[i - 1, :-1] + D[i - 1, :-1]))
        I[i, 1:] = p["mi"][r] * M[i - 1, 1:] + p["ii"][r] * I[i - 1, 1:]
        for j in range(1, H + 1):
            D[i, j] = p["md"][r] * M[i, j - 1] + p["dd"][r] * D[i, j - 1]
    return M, I, D


def scaled_sweep(read, hap, p, init, rows):
    """The scaled form over `rows` >= L rows (uniform priors: row 0's)."""
    L, H = len(read), len(hap)
    mi, gapm, mm, ii, dd = (float(p[k][0]) for k in ("mi", "gapm", "mm", "ii", "dd"))
    c = mi * gapm
    E = np.zeros((rows, H))
    E[:L] = emissions(read, hap, p) * c
    iis = np.array([ii if r < L else (mi if r == L else 1.0) for r in range(rows)])
    Mp = np.zeros(H + 1); Ip = np.zeros(H + 1); Dp = np.full(H + 1, init); Dp[0] = 0.0
    for r in range(rows):
        M = np.zeros(H + 1); I = np.zeros(H + 1); D = np.zeros(H + 1)
        M[1:] = E[r] * ((mm / c) * Mp[:-1] + Ip[:-1] + Dp[:-1])
        I[1:] = iis[r] * Ip[1:] + Mp[1:]
        for j in range(1, H + 1):
            D[j] = dd * D[j - 1] + M[j - 1]
        Mp, Ip, Dp = M, I, D
    last_is_pass_through = L < rows
    if last_is_pass_through:
        return Ip[1:].sum() / mi
    return Mp[1:].sum() / mi + Ip[1:].sum()


def random_pair(rng, L, H, uniform):
    hap = rng.integers(0, 4, H)
    start = int(rng.integers(0, max(1, H - L + 1)))
    read = hap[start:start + L].copy() if H >= L else rng.integers(0, 4, L)
    flip = rng.random(L) < 0.05
    read[flip] = (read[flip] + 1) % 4
    q = rng.integers(10, 41, L)
    if uniform:
        ins = dele = np.full(L, 45); gcp = np.full(L, 10)
    else:
        ins, dele, gcp = (rng.integers(8, 46, L) for _ in range(3))
    return read, hap, priors(q, ins, dele, gcp)


@pytest.mark.parametrize("L,rows", [(20, 32), (32, 32), (45, 64), (64, 64), (70, 96)])
def test_scaled_form_equals_the_reference_recurrence(L, rows):
    rng = np.random.default_rng(L * 100 + rows)
    for _ in range(4):
        H = int(rng.integers(max(2, L - 10), L + 40))
        read, hap, p = random_pair(rng, L, H, uniform=True)
        init = 2.0 ** 120 / H
        M, I, _ = reference_dp(read, hap, p, init)
        ref = M[L, 1:].sum() + I[L, 1:].sum()
        got = scaled_sweep(read, hap, p, init, rows)
        assert ref > 0
        assert abs(got - ref) <= 1e-12 * ref, (L, rows, got, ref)


@pytest.mark.parametrize("uniform", [True, False])
def test_row_sums_bound_the_likelihood(uniform):
    rng = np.random.default_rng(5 if uniform else 6)
    for _ in range(8):
        L = int(rng.integers(5, 60)); H = int(rng.integers(5, 90))
        read, hap, p = random_pair(rng, L, H, uniform)
        M, I, _ = reference_dp(read, hap, p, 1.0)
        lik = M[L, 1:].sum() + I[L, 1:].sum()
        for r in range(1, L + 1):
            bound = M[r, 1:].sum() + I[r, 1:].sum()
            assert lik <= bound * (1 + 1e-12), (r, lik, bound)


# ---- float32 chain sweep: the sum row against a running sum -----------------
#
# The chain kernels sweep one read (per f32x2 half) across several
# haplotypes laid end to end with a separator column between them (emission
# 0 in every row; each row's D cleared after it).  Below the read's rows sit
# pass-through rows (emission 0; ii = mi on the first, 1 below), so the last
# row carries the value whose column sum per haplotype is the result.  The
# kernels once added that value into a running sum every step; now the last
# row is a sum row with emission 1 for every code, and D takes each row's ii,
# so the sum row's M is the value one column back and its D = D + M the sum
# of the earlier columns: D + M at the separator column is the haplotype's
# sum.  Emulated in float32 with one rounding per operation (as the kernels'
# .rn PTX), the two must give bitwise the same sums.

def _f32(x):
    return np.float32(x)


def _fma(a, b, c):
    return np.float32(np.float64(a) * np.float64(b) + np.float64(c))


def _mul(a, b):
    return np.float32(np.float64(a) * np.float64(b))


def _add(a, b):
    return _fma(1.0, a, b)


def chain_sweep_f32(read, haps, p, init, rows, sum_row):
    """Per-haplotype parked sums of a float32 scaled chain sweep."""
    L = len(read)
    mi, gapm, mm, ii, dd = (float(p[k][0]) for k in ("mi", "gapm", "mm", "ii", "dd"))
    c = mi * gapm
    mmc = _f32(mm / c)
    iis = [_f32(ii) if r < L else (_f32(mi) if r == L else _f32(1.0)) for r in range(rows)]
    ddU = _f32(dd)
    # emission rows of every column of the chain (None: separator column)
    cols = []
    for k, hap in enumerate(haps):
        E = (emissions(read, hap, p) * c).astype(np.float32)
        for j in range(len(hap)):
            cols.append(E[:, j])
        cols.append(None)
    M = [_f32(0)] * rows; I = [_f32(0)] * rows; D = [_f32(0)] * rows
    acc = _f32(0)
    parked = []
    for col in cols:
        e = [_f32(0)] * rows
        if col is not None:
            e[:L] = [_f32(v) for v in col]
        if sum_row:
            e[rows - 1] = _f32(1.0)
        oM, oI, oD = M, I, D
        M = [None] * rows; I = [None] * rows; D = [None] * rows
        for r in range(rows):
            if r == 0:
                t = _f32(init)              # row 0's boundary, D^ = init
                I[0] = _f32(0)
            else:
                t = _fma(mmc, oM[r - 1], _add(oI[r - 1], oD[r - 1]))
                I[r] = _fma(iis[r], I[r - 1], M[r - 1])
            M[r] = _mul(t, e[r])
            D[r] = _fma(iis[r] if sum_row else ddU, oD[r], oM[r])
        if not sum_row:
            acc = _add(acc, I[rows - 1])
        if col is None:                     # a separator column
            if sum_row:
                parked.append(_add(D[rows - 1], M[rows - 1]))
                M[rows - 1] = _f32(0)
            else:
                parked.append(acc)
                acc = _f32(0)
            D = [_f32(0)] * rows
    return parked


@pytest.mark.parametrize("L,rows", [(12, 16), (14, 16), (15, 18), (30, 40)])
def test_sum_row_gives_the_running_sum_bitwise(L, rows):
    rng = np.random.default_rng(L * 7 + rows)
    haps = [rng.integers(0, 4, int(rng.integers(L // 2, 2 * L))) for _ in range(3)]
    read = haps[0][:L].copy() if len(haps[0]) >= L else rng.integers(0, 4, L)
    read[rng.random(L) < 0.1] = 0
    p = priors(rng.integers(10, 41, L), np.full(L, 45), np.full(L, 45), np.full(L, 10))
    init = 2.0 ** 120 / max(len(h) for h in haps)
    old = chain_sweep_f32(read, haps, p, init, rows, sum_row=False)
    new = chain_sweep_f32(read, haps, p, init, rows, sum_row=True)
    assert len(old) == len(new) == len(haps)
    for a, b in zip(old, new):
        assert a.tobytes() == b.tobytes(), (a, b)
    # and both are the likelihood (times mi) of each haplotype's own DP, with
    # row 0's D = init in every column, column 0 included (the reference's
    # initialisation, which the sweeps apply as row 0's M term at every step;
    # reference_dp above leaves column 0 at zero for the algebra tests)
    for h, got in zip(haps, new):
        H = len(h)
        E = emissions(read, h, p)
        M = np.zeros((L + 1, H + 1)); I = np.zeros_like(M); D = np.zeros_like(M)
        D[0, :] = init
        for i in range(1, L + 1):
            r = i - 1
            M[i, 1:] = E[r] * (p["mm"][r] * M[i - 1, :-1] +
                               p["gapm"][r] * (I[i - 1, :-1] + D[i - 1, :-1]))
            I[i, 1:] = p["mi"][r] * M[i - 1, 1:] + p["ii"][r] * I[i - 1, 1:]
            for j in range(1, H + 1):
                D[i, j] = p["md"][r] * M[i, j - 1] + p["dd"][r] * D[i, j - 1]
        ref = (M[L, 1:].sum() + I[L, 1:].sum()) * float(p["mi"][0])
        assert ref > 0
        assert abs(float(got) - ref) <= 2e-4 * ref, (float(got), ref)
