"""Host emulations of the index logic of two EMI kernels, run before their first GPU use:
the pivot-pair symmetric sweep (thread ownership of the lower triangle, the fix-ups of the
pivot rows and columns, the columns published for the next pair; `sweep_pair` and
`sweep_publish` in moraine_b200/csrc/emi_fast.cu) and the reduction's decode of the
upper-packed inverse index. Pure Python on the CPU; the CUDA kernels themselves are checked
on the GPU by tests/test_gpu_parity.py."""
import numpy as np
import pytest


def lt(ib, jb):
    return ib * (ib + 1) // 2 + jb


def sweep_pairs(A0, n, NB):
    """inv(A0) by the pivot-pair sweep with the kernel's 16 x 16 thread ownership."""
    N16 = 16 * NB
    A = np.eye(N16)
    A[:n, :n] = A0
    a = np.zeros((16, 16, NB * (NB + 1) // 2))  # a[ty, tx]: the thread's lower-triangle values
    for ty in range(16):
        for tx in range(16):
            for ib in range(NB):
                for jb in range(ib + 1):
                    i, j = ty + 16 * ib, tx + 16 * jb
                    a[ty, tx, lt(ib, jb)] = A[i, j] if i >= j else 0.0
    col = np.full((2, N16, 2), np.nan)

    def publish(k2, out):
        kbx, kt2 = k2 >> 4, k2 & 15
        for ty in range(16):
            for tx in range(16):
                if tx in (kt2, kt2 + 1):
                    c = tx - kt2
                    for ib in range(kbx, NB):
                        i = ty + 16 * ib
                        if i >= k2 + c:
                            out[i, c] = a[ty, tx, lt(ib, kbx)]
                if ty in (kt2, kt2 + 1):
                    r = ty - kt2
                    for jb in range(kbx + 1):
                        j = tx + 16 * jb
                        if j < k2 + r:
                            out[j, r] = a[ty, tx, lt(kbx, jb)]

    publish(0, col[0])
    small = False
    for k in range(0, n, 2):
        KB, kt, buf = k >> 4, k & 15, (k >> 1) & 1
        c = col[buf].copy()
        assert not np.isnan(c).any(), "a published column entry was never written"
        p00, p10, p11 = c[k, 0], c[k, 1], c[k + 1, 1]
        assert c[k + 1, 0] == p10
        r0 = 1.0 / (p00 if p00 != 0 else 1.0)
        t = p10 * r0
        d1 = p11 - t * p10
        r1 = 1.0 / (d1 if d1 != 0 else 1.0)
        small |= not (abs(p00) >= 1e-9 and abs(d1) >= 1e-9)
        for ty in range(16):
            for tx in range(16):
                cj = [(c[tx + 16 * jb, 0], c[tx + 16 * jb, 1] - t * c[tx + 16 * jb, 0]) for jb in range(NB)]
                colk = tx in (kt, kt + 1)
                for ib in range(NB):
                    ci = c[ty + 16 * ib]
                    g0, g1 = ci[0] * r0, (ci[1] - t * ci[0]) * r1
                    for jb in range(ib + 1):
                        v = a[ty, tx, lt(ib, jb)]
                        v -= g0 * cj[jb][0]
                        v -= g1 * cj[jb][1]
                        if jb == KB and colk:
                            v = g0 - t * g1 if tx == kt else g1
                        a[ty, tx, lt(ib, jb)] = v
                if ty in (kt, kt + 1):
                    row1 = ty != kt
                    for jb in range(KB + 1):
                        g0, g1 = cj[jb][0] * r0, cj[jb][1] * r1
                        w = g1 if row1 else g0 - t * g1
                        if jb == KB and colk:
                            w = (t * r1 if tx == kt else -r1) if row1 else (-(r0 + t * t * r1) if tx == kt else t * r1)
                        a[ty, tx, lt(KB, jb)] = w
        if k + 2 < n:
            col[buf ^ 1][:] = np.nan
            publish(k + 2, col[buf ^ 1])
    inv = np.zeros((n, n))
    for ty in range(16):
        for tx in range(16):
            for ib in range(NB):
                for jb in range(ib + 1):
                    i, j = ty + 16 * ib, tx + 16 * jb
                    if i < n and j <= i:
                        inv[i, j] = inv[j, i] = -a[ty, tx, lt(ib, jb)]
    return inv, small


@pytest.mark.parametrize("n", [2, 3, 5, 16, 17, 31, 33])
def test_pivot_pair_sweep_index_logic(n):
    """Every published entry is written, every owner's value ends as -inv, with odd n through
    the identity padding, on an indefinite |Gamma| of coherence magnitudes."""
    rng = np.random.default_rng(n)
    x = rng.normal(size=(n, n + 4)) + 1j * rng.normal(size=(n, n + 4))
    g = x @ x.conj().T
    d = np.sqrt(np.diag(g).real)
    G = np.abs(g / np.outer(d, d))
    inv, small = sweep_pairs(G, n, max(2, (n + 15) // 16))
    ref = np.linalg.inv(G)
    assert not small
    assert np.abs(inv - ref).max() <= 50 * np.finfo(float).eps * np.linalg.cond(G) * np.abs(ref).max()


def test_pivot_pair_sweep_flags_a_small_pivot():
    n = 6
    G = np.full((n, n), 0.3) + np.eye(n) * 0.7
    G[0, 1] = G[1, 0] = 1 - 1e-12  # second natural-order pivot ~2e-12
    _, small = sweep_pairs(G, n, 2)
    assert small


def tri_up(m, j, n):
    return m * n - m * (m - 1) // 2 + (j - m)


@pytest.mark.parametrize("n", list(range(2, 129)))
def test_upper_packed_decode(n):
    """The reduction's walk from a packed index q to its row m (bounded by the last row, so it
    ends for threads past the last entry, N <= 21 included) agrees with a direct decode."""
    np_ = n * (n + 1) // 2
    for tid in range(256):
        m = 0
        while m + 1 < n and tri_up(m + 1, m + 1, n) <= tid:
            m += 1
        for q in range(tid, np_, 256):
            while m + 1 < n and tri_up(m + 1, m + 1, n) <= q:
                m += 1
            j = m + (q - tri_up(m, m, n))
            mm = max(r for r in range(n) if tri_up(r, r, n) <= q)
            assert (m, j) == (mm, mm + q - tri_up(mm, mm, n)) and m <= j < n
