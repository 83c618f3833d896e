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


# ---- k_dct_tma: 128B-swizzled 16-column tiles, warp w owns chunk w ----------

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
