"""Host-side check of the det-128 ptycho kernels' two-exchange transform.

The kernels `k_ptycho_fwd128` / `k_ptycho_adj128` (csrc/pt_ptycho.cu)
compute B[u][v] = f sum_{r,q} A[r][q] w^(DIR (u r + v q)), w = exp(2 pi i /
128), in three register rounds with two trips through a 128 KB shared buffer:

  R1  thread (q = tid & 127, rt = (tid >> 7) + 4 c): 16-point DFT over m of
      r = rt + 8 m, times w^(rt k1), written to E1[k1][qa][rt][qb]
  R2  thread (k1 = warp, qb = lane): 8-point DFT over rt (u = k1 + 16 k2),
      4-point DFT over qa of q = qb + 32 qa (v1), times w^(qb v1) f, written
      to E2[v1][u][qb] with 16-byte slots XOR-permuted by u & 7
  R3  thread (u = tid & 127, v1 = tid >> 7): 32-point DFT over qb,
      v = v1 + 4 v2.

This test restates the index maps of e1_at / e2_at and the thread roles,
checks that both exchange layouts are bijections onto the buffer, that
every warp-wide exchange access takes the minimum number of shared-memory
wavefronts (32 banks of 4 bytes), and that the rounds compute the 2-D DFT in
the orientation the kernels store (frame[kx][ky] for the forward, pixel
[y][x] for the adjoint).  No GPU is needed.
"""
import numpy as np

N = 128


def e1_at(k1, qa, rt, qb):
    return ((k1 * 4 + qa) * 8 + rt) * 32 + qb


def e2_at(v1, u, qb):
    return (v1 * 128 + u) * 32 + 2 * ((qb >> 1) ^ (u & 7)) + (qb & 1)


def wavefronts(byte_addrs, size):
    """Shared-memory wavefronts of one warp access: the most distinct 4-byte
    words that fall in any one of the 32 banks."""
    banks = {}
    for a in byte_addrs:
        for o in range(0, size, 4):
            word = (a + o) // 4
            banks.setdefault(word % 32, set()).add(word)
    return max(len(s) for s in banks.values())


def test_exchange_layouts_are_bijections():
    k1, qa, rt, qb = np.meshgrid(np.arange(16), np.arange(4), np.arange(8), np.arange(32), indexing="ij")
    e1 = e1_at(k1, qa, rt, qb).ravel()
    assert np.array_equal(np.sort(e1), np.arange(N * N))
    v1, u, qb = np.meshgrid(np.arange(4), np.arange(128), np.arange(32), indexing="ij")
    e2 = e2_at(v1, u, qb).ravel()
    assert np.array_equal(np.sort(e2), np.arange(N * N))


def test_exchange_accesses_take_minimum_wavefronts():
    # R1 writes (8 bytes): warp w, lanes = 32 consecutive q, fixed (c, k1)
    worst = 0
    for w in range(16):
        tids = np.arange(32 * w, 32 * w + 32)
        q = tids & 127
        for c in range(2):
            rt = (tids >> 7) + 4 * c
            for k1 in range(16):
                worst = max(worst, wavefronts(8 * e1_at(k1, q >> 5, rt, q & 31), 8))
    assert worst == 2
    # R2 reads of E1 (8 bytes) and writes of E2 (8 bytes): lanes = qb
    qb = np.arange(32)
    worst_r = max(wavefronts(8 * e1_at(k1, qa, rt, qb), 8)
                  for k1 in range(16) for qa in range(4) for rt in range(8))
    worst_w = max(wavefronts(8 * e2_at(v1, k1 + 16 * k2, qb), 8)
                  for k1 in range(16) for v1 in range(4) for k2 in range(8))
    assert worst_r == 2 and worst_w == 2
    # R3 reads of E2 (16 bytes): lanes = 32 consecutive u, slot s ^ (u & 7)
    worst = 0
    for w in range(16):
        tids = np.arange(32 * w, 32 * w + 32)
        u, v1 = tids & 127, tids >> 7
        for s in range(16):
            worst = max(worst, wavefronts(16 * ((v1 * 128 + u) * 16 + (s ^ (u & 7))), 16))
    assert worst == 4


def rounds(A, DIR, f):
    """The three rounds, vectorised over threads; returns B[u][v]."""
    w = lambda L, e: np.exp(DIR * 2j * np.pi * e / L)
    ex = np.full(N * N, np.nan, complex)
    # R1: rows r = rt + 8 m; 16-point DFT over m at each (rt, q)
    Ar = A.reshape(16, 8, N)                                  # [m][rt][q]
    m, k = np.arange(16)[:, None], np.arange(16)[None, :]
    R1 = np.einsum("mtq,mk->ktq", Ar, w(16, m * k))            # [k1][rt][q]
    R1 *= w(128, np.arange(16)[:, None, None] * np.arange(8)[None, :, None])
    k1, rt, q = np.meshgrid(np.arange(16), np.arange(8), np.arange(N), indexing="ij")
    ex[e1_at(k1, q >> 5, rt, q & 31)] = R1
    # R2: thread (k1, qb) reads (qa, rt)
    k1, qa, rt, qb = np.meshgrid(np.arange(16), np.arange(4), np.arange(8), np.arange(32), indexing="ij")
    a = ex[e1_at(k1, qa, rt, qb)]                              # [k1][qa][rt][qb]
    t, k2 = np.arange(8)[:, None], np.arange(8)[None, :]
    a = np.einsum("iatb,tk->iakb", a, w(8, t * k2))            # 8-point over rt -> k2
    g, v1 = np.arange(4)[:, None], np.arange(4)[None, :]
    a = np.einsum("iakb,av->ivkb", a, w(4, g * v1))            # 4-point over qa -> v1
    a *= f * w(128, np.arange(4)[None, :, None, None] * np.arange(32)[None, None, None, :])
    ex2 = np.full(N * N, np.nan, complex)
    k1, v1, k2, qb = np.meshgrid(np.arange(16), np.arange(4), np.arange(8), np.arange(32), indexing="ij")
    ex2[e2_at(v1, k1 + 16 * k2, qb)] = a
    # R3: thread (u, v1) reads qb, 32-point DFT -> v = v1 + 4 v2
    v1, u, qb = np.meshgrid(np.arange(4), np.arange(N), np.arange(32), indexing="ij")
    b = ex2[e2_at(v1, u, qb)]                                  # [v1][u][qb]
    s, v2 = np.arange(32)[:, None], np.arange(32)[None, :]
    b = np.einsum("vus,sk->vuk", b, w(32, s * v2))             # [v1][u][v2]
    B = np.empty((N, N), complex)
    for j in range(4):
        B[:, j::4] = b[j]                                      # v = v1 + 4 v2
    return B


def test_rounds_compute_the_frame_transforms():
    rng = np.random.default_rng(0)
    f = 0.3 * np.exp(0.7j)
    F = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))   # probe x patch [y][x]
    B = rounds(F, -1, f)                                                 # B[u = ky][v = kx]
    frame = B.T                                                          # stored frame[kx][ky]
    ref = f * np.fft.fft2(F).T
    assert np.abs(frame - ref).max() <= 1e-10 * np.abs(ref).max()
    G = rng.standard_normal((N, N)) + 1j * rng.standard_normal((N, N))   # frame[kx][ky]
    S = rounds(G, +1, f).T                                               # pixel [y][x]
    ref = f * np.fft.ifft2(G.T) * N * N
    assert np.abs(S - ref).max() <= 1e-10 * np.abs(ref).max()
