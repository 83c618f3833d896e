"""The shared-memory index maps of the transform kernels (no GPU).

The maps are restated from `vring_b200/csrc/vr_poisson.cu`. The tests check
that they are bijections on the buffers they permute. They also check that
every 16-byte access pattern the kernels issue is bank-conflict-free: shared
memory serves a warp's 16-byte accesses one quarter warp (8 lanes, 128
bytes) at a time, so each quarter warp must touch 8 distinct 16-byte bank
groups.

Where a pattern is knowingly not conflict-free, the test pins its conflict
degree instead, so that a change shows up here.
"""


def brev(x, bits):
    r = 0
    for i in range(bits):
        r |= ((x >> i) & 1) << (bits - 1 - i)
    return r


def quarter_warp_degree(chunks):
    """Worst number of distinct 16-byte words that share a bank group within
    one quarter warp (1 = conflict-free; equal addresses are broadcast)."""
    worst = 1
    for qw in range(4):
        words = chunks[8 * qw:8 * qw + 8]
        by_group = {}
        for wd in set(words):
            by_group.setdefault(wd % 8, set()).add(wd)
        worst = max(worst, max(len(v) for v in by_group.values()))
    return worst


# ---- warp_fft512 (the slab kernels): 128B-swizzled 16-column tiles, warp w owns chunk w

def swz_word(r, w):
    """16-byte word of (row r, chunk w) in a 128B-swizzled tile (swz_pair)."""
    return r * 8 + (w ^ (r & 7))


def scratch0_row(k):
    return k ^ (((k >> 5) & 3) << 1)


def scratch1_row(k):
    return k ^ (((k >> 8) & 1) << 2)


def test_dct_scratch_rows_are_permutations():
    assert sorted(scratch0_row(k) for k in range(512)) == list(range(512))
    assert sorted(scratch1_row(k) for k in range(512)) == list(range(512))


def test_dct_fft_transpose_is_conflict_free():
    for w in range(8):
        for k1 in range(16):  # writes: entry t + 32 k1 from lane t
            words = [swz_word(scratch0_row(t + 32 * k1), w) for t in range(32)]
            assert quarter_warp_degree(words) == 1
        for u in range(16):  # reads: entry 2u + h + 32 k1, k1 = lane / 2, h = lane & 1
            words = [swz_word(scratch0_row(2 * u + (l & 1) + 32 * (l >> 1)), w) for l in range(32)]
            assert quarter_warp_degree(words) == 1


def test_dct_output_scratch_is_conflict_free():
    for w in range(8):
        for q in range(16):  # FFT output writes
            words = [swz_word(scratch1_row((l >> 1) + 16 * (16 * (l & 1) + brev(q, 4))), w) for l in range(32)]
            assert quarter_warp_degree(words) == 1
            ks = [l + 32 * q for l in range(32)]  # reads of k and 512 - k
            assert quarter_warp_degree([swz_word(scratch1_row(k), w) for k in ks]) == 1
            km = [swz_word(scratch1_row((512 - k) & 511), w) for k in ks]
            # 512 - k meets a block of 8 rows on both sides of 256 only for
            # q = 0 (k = 0 maps to 0) and q = 8 (k = 256 maps to 256): 2-way there
            assert quarter_warp_degree(km) == (2 if q in (0, 8) else 1)


def test_dct_data_rows_degree():
    # true data rows: Makhoul's input read 2n / 2(N-1-n)+1 is 2-way, the
    # backward output write and the k = lane + 32 q accesses are conflict-free
    N = 512
    for w in range(8):
        for q in range(16):
            src = [2 * n if n < N // 2 else 2 * (N - 1 - n) + 1 for n in (l + 32 * q for l in range(32))]
            assert quarter_warp_degree([swz_word(r, w) for r in src]) == 2
            assert quarter_warp_degree([swz_word(l + 32 * q, w) for l in range(32)]) == 1
            outs = []
            for l in range(32):
                m = (l >> 1) + 16 * (16 * (l & 1) + brev(q, 4))
                outs.append(swz_word(2 * m if m < N // 2 else 2 * (N - 1 - m) + 1, w))
            assert quarter_warp_degree(outs) == 1


# ---- k_fft_fwd_s / k_fft_bwd_s: pairs of lines as 16-byte words -------------

def pair_stride(T):
    return 16 * T + (T if T < 8 else 0)


def fft_swz(T, k):
    G = 16 // T
    return (k // G) & ((T if T < 8 else 8) - 1)


def fft_word(T, pl, k, c):
    """16-byte word of transpose entry (row k, column c) of pair pl."""
    return 15 * T + pl * pair_stride(T) + k * T + (c ^ fft_swz(T, k))


def test_fft_transpose_map_is_a_permutation():
    for T in (2, 4, 8, 16):
        cells = sorted(k * T + (c ^ fft_swz(T, k)) for k in range(16) for c in range(T))
        assert cells == list(range(16 * T))


def test_fft_transpose_is_conflict_free():
    for T in (2, 4, 8, 16):
        G = 16 // T
        lanes = [(l // T, l % T) for l in range(32)]  # (pair of the warp, thread t)
        for wp in range(4):  # a block's warps hold consecutive pairs
            base = wp * (32 // T)
            for k1 in range(16):  # writes: row k1, column t
                words = [fft_word(T, base + pl, k1, t) for pl, t in lanes]
                assert quarter_warp_degree(words) == 1, (T, k1)
            for u in range(G):  # reads: row t G + u, column tt
                for tt in range(T):
                    words = [fft_word(T, base + pl, t * G + u, tt) for pl, t in lanes]
                    assert quarter_warp_degree(words) == 1, (T, u, tt)


def fft_natural_word(T, pl, k):
    """16-byte word of entry k of pair pl in natural order (the transform's
    output and the inverse transform's staged input)."""
    return 15 * T + pl * pair_stride(T) + k


def packed_slot(T, n):
    return n ^ ((n >> 3) & 1) if T == 8 else n


def test_fft_natural_order_write_is_conflict_free_at_128():
    # pair_fft16's last write, k = 2 t + u + 16 k2: the lanes t >= 4 of a
    # pair write the other u in the same instruction; with the same u in
    # every lane it would be 2-way
    T, G = 8, 2
    lanes = [(l // T, l % T) for l in range(32)]
    for u0 in range(G):
        for k2 in range(T):
            words = [fft_natural_word(T, pl, t * G + (u0 ^ int(t >= 4)) + 16 * k2) for pl, t in lanes]
            assert quarter_warp_degree(words) == 1
            same_u = [fft_natural_word(T, pl, t * G + u0 + 16 * k2) for pl, t in lanes]
            assert quarter_warp_degree(same_u) == 2
    # every entry is written exactly once
    for t in range(T):
        ks = sorted(t * G + (u0 ^ int(t >= 4)) + 16 * k2 for u0 in range(G) for k2 in range(T))
        assert ks == sorted(t * G + u + 16 * k2 for u in range(G) for k2 in range(T))


def test_fft_forward_output_reads_are_conflict_free():
    T, N = 8, 128
    lanes = [(l // T, l % T) for l in range(32)]
    for jj in range(N // (2 * T)):
        ks = [(pl, t + T * jj) for pl, t in lanes]
        assert quarter_warp_degree_active([fft_natural_word(T, pl, k) if k else None for pl, k in ks]) == 1
        assert quarter_warp_degree_active([fft_natural_word(T, pl, N - k) if k else None for pl, k in ks]) == 1


def quarter_warp_degree_active(words):
    """quarter_warp_degree over the lanes that take part (None: the lane
    issues its access in another branch)."""
    worst = 1
    for qw in range(4):
        by_group = {}
        for wd in set(w for w in words[8 * qw:8 * qw + 8] if w is not None):
            by_group.setdefault(wd % 8, set()).add(wd)
        if by_group:
            worst = max(worst, max(len(v) for v in by_group.values()))
    return worst


def test_fft_inverse_packed_staging_is_conflict_free_at_128():
    T, N = 8, 128
    assert sorted(packed_slot(T, n) for n in range(N)) == list(range(N))
    lanes = [(l // T, l % T) for l in range(32)]
    for j in range(16):  # staging writes of entries t + T j
        assert quarter_warp_degree([fft_natural_word(T, pl, packed_slot(T, t + T * j)) for pl, t in lanes]) == 1
    for m in range(16):  # reads of entries 2 kk - 1 and 2 kk
        kks = [(pl, (t + T * m) if t + T * m <= N // 2 else N - (t + T * m)) for pl, t in lanes]
        odd = [fft_natural_word(T, pl, packed_slot(T, 2 * kk - 1)) if kk > 0 else None for pl, kk in kks]
        even = [fft_natural_word(T, pl, packed_slot(T, 2 * kk)) if 0 < 2 * kk < N else None for pl, kk in kks]
        assert quarter_warp_degree_active(odd) == 1, m
        assert quarter_warp_degree_active(even) == 1, m
        plain = [fft_natural_word(T, pl, 2 * kk) if 0 < 2 * kk < N else None for pl, kk in kks]
        assert quarter_warp_degree_active(plain) == 2  # the unpermuted layout


# ---- k_dct_tma: two warps per column pair, N = 8 x 8 x 8 ----------------------
# thread u = lane + 32 h of pair p (warps 2p, 2p + 1) owns chunk p of each row

def pfft_k2(u):
    return ((u >> 5) << 2) | (u & 3)


def pfft_c(u):
    return (u >> 2) & 7


def pfft_r2(k2, a, c):
    return 64 * k2 + 8 * c + (a ^ (((k2 & 3) << 1) | (c & 1)))


def pfft_p(m):
    return m ^ (((m >> 3) & 1) << 2)


def mk_row(n):
    return 2 * n if n < 256 else 1023 - 2 * n


def pair_degree(row_of_u, p):
    """worst quarter-warp degree over the two warps of pair p"""
    return max(quarter_warp_degree([swz_word(row_of_u(l + 32 * h), p) for l in range(32)]) for h in range(2))


def test_pair_fft_maps_are_permutations():
    assert sorted(64 * k2 + n1 for k2 in range(8) for n1 in range(64)) == list(range(512))
    assert sorted(pfft_r2(k2, a, c) for k2 in range(8) for a in range(8) for c in range(8)) == list(range(512))
    assert sorted(pfft_p(m) for m in range(512)) == list(range(512))
    assert sorted(mk_row(n) for n in range(512)) == list(range(512))
    # after the FFT every (k2, c) is held by exactly one thread
    assert sorted(pfft_k2(u) + 8 * pfft_c(u) for u in range(64)) == list(range(64))


def test_pair_fft_transposes_are_conflict_free():
    for p in range(8):
        for k2 in range(8):  # writes: entry (n1 = u, k2) at row 64 k2 + n1
            assert pair_degree(lambda u: 64 * k2 + u, p) == 1
        for b in range(8):  # reads by thread (k2, a) = (u / 8, u % 8) of entry (a + 8 b, k2)
            assert pair_degree(lambda u: 64 * (u >> 3) + (u & 7) + 8 * b, p) == 1
        for c in range(8):  # second transpose, writes by thread (u / 8, u % 8)
            assert pair_degree(lambda u: pfft_r2(u >> 3, u & 7, c), p) == 1
        for a in range(8):  # reads by thread (pfft_k2, pfft_c)
            assert pair_degree(lambda u: pfft_r2(pfft_k2(u), a, pfft_c(u)), p) == 1


def test_pair_dct_data_rows_degree():
    for p in range(8):
        for q in range(4):  # forward loads: lanes with u & 4 take slot q + 4 first
            assert pair_degree(lambda u: mk_row(u + 64 * (q + 4 if (u >> 2) & 1 else q)), p) == 1
            assert pair_degree(lambda u: mk_row(u + 64 * (q if (u >> 2) & 1 else q + 4)), p) == 1
            # without the swap the even rows 2n would be 2-way
            assert pair_degree(lambda u: mk_row(u + 64 * q), p) == 2
        for d in range(8):  # forward: X[m] to scratch row pfft_p(m)
            assert pair_degree(lambda u: pfft_p(pfft_k2(u) + 8 * pfft_c(u) + 64 * d), p) == 1
        for q in range(8):
            assert pair_degree(lambda u: pfft_p(u + 64 * q), p) == 1
            # the partner rows 512 - k cross a block of 8 rows: 2-way
            assert pair_degree(lambda u: pfft_p((512 - u - 64 * q) & 511), p) == 2
            assert pair_degree(lambda u: u + 64 * q, p) == 1  # results; inverse loads of k
            assert pair_degree(lambda u: (512 - u - 64 * q) & 511, p) == 1  # inverse loads of 512 - k
        for j in range(8):  # inverse outputs: lanes with odd c take slot j ^ 4 first
            def row(u):
                d = j ^ 4 if pfft_c(u) & 1 else j
                return mk_row(pfft_k2(u) + 8 * pfft_c(u) + 64 * d)
            assert pair_degree(row, p) == 1


def test_pair_fft_decomposition_matches_numpy():
    # the three radix-8 stages with the kernel's index maps, each 8-point DFT
    # leaving X[k] in slot brev3(k), against numpy's FFT
    import numpy as np
    N = 512
    W = lambda e, n: np.exp(-2j * np.pi * e / n)

    def dft8(v):
        X = np.fft.fft(v)
        out = np.empty(8, complex)
        for k in range(8):
            out[brev(k, 3)] = X[k]
        return out

    rng = np.random.default_rng(3)
    x = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    scratch = np.empty(N, complex)
    for u in range(64):
        y = dft8(x[u + 64 * np.arange(8)])
        for k2 in range(8):
            scratch[64 * k2 + u] = y[brev(k2, 3)] * W(u * k2, 512)
    mid = {}
    for u in range(64):
        k2, a = u >> 3, u & 7
        mid[u] = dft8(np.array([scratch[64 * k2 + a + 8 * b] for b in range(8)]))
    for u in range(64):
        k2, a = u >> 3, u & 7
        for c in range(8):
            scratch[pfft_r2(k2, a, c)] = mid[u][brev(c, 3)] * W(a * c, 64)
    X = np.empty(N, complex)
    for u in range(64):
        k2, c = pfft_k2(u), pfft_c(u)
        z = dft8(np.array([scratch[pfft_r2(k2, a, c)] for a in range(8)]))
        for d in range(8):
            X[k2 + 8 * c + 64 * d] = z[brev(d, 3)]
    ref = np.fft.fft(x)
    assert np.abs(X - ref).max() <= 1e-13 * np.abs(ref).max()
