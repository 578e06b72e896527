"""CPU replay of the index arithmetic of the 3-D mixed-precision step's kernels.

A 3-D run holds its state as the DFT along n in two layouts of L*M*Hp complex floats per
array (Hp = N/2 + 1 rounded up to the tile width CT, Tn = Hp/CT n-tiles):
  layout A (row view, rows l*M + m of length N):  ((t*L + l)*M + m)*CT + c
  layout B (column view, (t, km) tiles of L rows): ((t*M + km)*L + l)*CT + c
Each kernel's global and shared accesses are replayed here with numpy, from the same
formulas as the kernels (csrc/mrow_kernel.cuh: ROW_TILE_LOOP, build_pair_d, the step's
pointwise and forward stores; csrc/step_3d.cu: k_mpass; csrc/mcol_kernel.cuh:
k_mcol_step's items, tiles, table planes and k-vector reads), and checked: every index
inside the buffer it addresses, the row walk visiting each (row, kn <= N/2) once, the
m-axis passes mapping layout A onto layout B one to one, the shared buffers inside
the CTA's dynamic shared memory, and the checkpoint column kernel's gradient partials
covering each spectral column once, from rows that do not depend on the tile width.  The grid shapes include the three on which an earlier,
since removed, 3-D build faulted at run creation.
"""
import numpy as np
import pytest

SMS = 148
MROW_TILE, MCOL_TILE, COL_TILE_MAX = 2048, 2048, 16


def spad(i):
    return i + (i >> 4)


def padded_len(n):
    return n + (n >> 4) + 1


def mcol_tile_ok(L, C):
    return 1 <= C <= COL_TILE_MAX and 512 <= C * L <= 4096


def tile_width_3d(L, M):
    """engine.cu tile_width_3d: the widest column tile width from the mixed default down
    that the column kernel (L x CT) and the m-axis pass (M x CT) both take."""
    d = max(1, min(COL_TILE_MAX, MCOL_TILE // L))
    cands = [c for c in (d // 4, d // 2, d, 2 * d) if c >= 1 and mcol_tile_ok(L, c)]
    c = d
    while c >= 1:
        if c in cands and M * c <= 4096:
            return c
        c //= 2
    return 0


def geometry(L, M, N):
    ct = tile_width_3d(L, M)
    hp = -(-(N // 2 + 1) // ct) * ct
    return ct, hp, hp // ct, L * M * hp


# the last two run at column tile widths 16 and 1 (the inverse m-axis pass's 8-byte copies)
SHAPES = [(64, 64, 32), (128, 128, 64), (256, 128, 64), (256, 256, 64), (32, 32, 8), (64, 128, 32), (128, 64, 16),
          (32, 64, 16), (2048, 32, 16)]


@pytest.mark.parametrize("L,M,N", SHAPES)
def test_row_kernels_stay_inside_layout_a(L, M, N):
    ct, hp, tn, E = geometry(L, M, N)
    assert ct >= 1
    R, H = L * M, N // 2
    lct = ct.bit_length() - 1
    rpc = max((MROW_TILE // 2) // N, min(2, 2048 // N), 1)  # mrow_rpc (step_common.cuh)
    lrpc = rpc.bit_length() - 1
    nt = min(2 * rpc * N // 16, 512)
    grid = -(-R // rpc)
    # ROW_TILE_LOOP over every CTA (vectorised over CTAs and w)
    lblk = lrpc + lct
    w = np.arange(tn << lblk)
    t, rem = w >> lblk, w & ((1 << lblk) - 1)
    r, k = rem >> lct, (t << lct) + (rem & (ct - 1))
    keep = k <= H
    r, k = r[keep], k[keep]
    l = (np.arange(grid)[:, None] * rpc + r[None, :]).ravel()
    kk = np.broadcast_to(k, (grid, k.size)).ravel()
    inside = l < R
    l, kk = l[inside], kk[inside]
    rs = ((kk >> lct) * R + l) * ct + (kk & (ct - 1))
    assert rs.min() >= 0 and rs.max() < E
    # each (row, kn <= N/2) exactly once
    assert np.array_equal(np.sort(l * (H + 1) + kk), np.arange(R * (H + 1)))
    # shared memory of the row step (NB = 2 RPC sequences) and of the analysis (3 RPC)
    for nb in (2 * rpc, 3 * rpc):
        b = np.arange(nb)
        kv = np.arange(H + 1)
        idx = np.concatenate([spad(kv[:, None] * nb + b[None, :]).ravel(),
                              spad(((N - kv[1:H])[:, None]) * nb + b[None, :]).ravel()])
        assert idx.max() < padded_len(nb * N)
    # the step's pointwise stores and forward-transform reads (RPC interleaved sequences)
    wv = np.arange(rpc * N)
    assert spad(wv).max() < padded_len(2 * rpc * N)
    kv, rv = np.arange(H + 1)[:, None], np.arange(rpc)[None, :]
    assert max(spad(kv * rpc + rv).max(), spad(((N - kv) & (N - 1)) * rpc + rv).max()) < padded_len(2 * rpc * N)
    # the analysis kernel's partial sums and the forward kernel's real-space reads
    assert 2 * (grid - 1) + 1 < 2 * grid
    assert (R - 1) * N + (N - 1) < L * M * N
    assert nt >= 32 and nt % 32 == 0


@pytest.mark.parametrize("L,M,N", SHAPES)
def test_m_axis_passes_map_layout_a_onto_layout_b(L, M, N):
    ct, hp, tn, E = geometry(L, M, N)
    assert M * ct <= 4096 and ct in (1, 2, 4, 8, 16)
    t, l, i = np.meshgrid(np.arange(tn), np.arange(L), np.arange(M * ct), indexing="ij")
    block_a = (t * L + l) * M * ct
    src_a = block_a + i  # the forward pass's float4 loads cover i < M*CT of the A block
    km, c = i // ct, i % ct
    dst_b = ((t * M + km) * L + l) * ct + c
    assert src_a.min() >= 0 and src_a.max() < E and dst_b.min() >= 0 and dst_b.max() < E
    # one to one in both directions (the inverse pass gathers B and stores the A block)
    assert np.array_equal(np.sort(src_a.ravel()), np.arange(E))
    assert np.array_equal(np.sort(dst_b.ravel()), np.arange(E))
    assert spad(M * ct - 1) < padded_len(M * ct)
    # the padded transform buffer, then the unpadded FP32 staging buffer (16-byte aligned)
    assert (16 * padded_len(M * ct)) % 16 == 0
    assert 16 * padded_len(M * ct) + 8 * M * ct <= 227 * 1024
    # the inverse pass's staged copies: CT-value chunks of B, 16-byte pieces when CT is even
    if ct >= 2:
        e = np.arange(0, M * ct, 2)
        src = ((0 * M + e // ct) * L + 0) * ct + e % ct
        assert (src % 2 == 0).all() and (e // ct == (e + 1) // ct).all()


@pytest.mark.parametrize("L,M,N", SHAPES)
def test_column_kernel_items_stay_inside_layout_b_and_tables(L, M, N):
    ct, hp, tn, E = geometry(L, M, N)
    T3 = tn * M
    nt = max(32, ct * L // 16)
    assert nt % ct == 0  # a thread's elements share one tile column
    smem = 2 * 16 * padded_len(ct * L) + 8 * ct * L + 8 * ct * L
    assert smem <= 227 * 1024
    fit = (228 * 1024) // (smem + 1024)
    minb = max(1, min(8, fit))
    items = T3  # one run
    g0 = min(items, minb * SMS)
    per = -(-items // g0)
    grid = -(-items // per)
    first = np.arange(grid) * per
    assert first.max() < items
    tiles = np.arange(items)
    lo, hi = tiles * L * ct, tiles * L * ct + L * ct - 1
    assert lo.min() >= 0 and hi.max() < E  # arrays and each table plane (T3*L*CT points)
    km3 = tiles % M
    kn = (tiles // M)[:, None] * ct + np.arange(ct)[None, :]
    assert km3.max() < M
    # k_n is read only where kn <= N/2 (past it the column is padding)
    assert kn[kn <= N // 2].max() < N
    # shared: the padded FFT buffers, then the FP32 staging buffer and the table slot
    e = np.arange(L * ct)
    assert spad(e).max() < padded_len(L * ct)
    q_off = 2 * 16 * padded_len(ct * L)
    t_off = q_off + 8 * L * ct
    assert q_off % 16 == 0 and t_off % 16 == 0 and (8 * L * ct) % 16 == 0
    # table planes: 4 planes of T3*L*CT doubles, 16-byte aligned tile starts
    assert (tiles * L * ct * 8 % 16 == 0).all()


def column_partials(L, M, N, ct, three_d):
    """The checkpoint column kernel's gradient partials (csrc/mcol_kernel.cuh, COL_STEP_CHECKPOINT):
    for each tile, thread b < C writes partial pair gpart_off + col for its column kc when
    kc <= hc; col = kc*M + km3 in the 3-D column view (tile t*M + km3, kc = t*CT + b, hc = N/2),
    col = kc in 2-D (tile t, kc = t*CT + b, hc = M/2).  Returns the written cols, and the
    per-thread sum's rows for every column (thread t_c*C + b takes rows t_c + j*L/16)."""
    nt = ct * L // 16
    if three_d:
        hp = -(-(N // 2 + 1) // ct) * ct
        tiles = (hp // ct) * M
        hc = N // 2
    else:
        hp = -(-(M // 2 + 1) // ct) * ct
        tiles = hp // ct
        hc = M // 2
    cols = []
    for tile in range(tiles):
        for b in range(ct):
            if three_d:
                kc, km3 = (tile // M) * ct + b, tile % M
                if kc <= hc:
                    cols.append(kc * M + km3)
            else:
                kc = tile * ct + b
                if kc <= hc:
                    cols.append(kc)
    rows = {}
    for tid in range(nt):
        b, tc = tid % ct, tid // ct
        rows[(b, tc)] = [(tid + j * nt) // ct for j in range((L * ct) // nt)]
        assert all((tid + j * nt) % ct == b for j in range((L * ct) // nt))
    return np.array(cols), rows, nt


@pytest.mark.parametrize("L,M,N", SHAPES)
def test_gradient_partials_cover_each_spectral_column_once_3d(L, M, N):
    ct, hp, tn, E = geometry(L, M, N)
    cols, rows, nt = column_partials(L, M, N, ct, True)
    gcols = (N // 2 + 1) * M  # engine.cu: the pairs allotted after the analysis partials
    assert len(cols) == gcols and np.array_equal(np.sort(cols), np.arange(gcols))
    # a column's threads take the same rows whatever the tile width: t_c + j*L/16
    for (b, tc), rr in rows.items():
        assert rr == [tc + j * (L // 16) for j in range(16)]


@pytest.mark.parametrize("L,M", [(64, 64), (256, 256), (1024, 1024), (32, 256), (2048, 64)])
def test_gradient_partials_do_not_depend_on_tile_width_2d(L, M):
    gcols = M // 2 + 1
    widths = [c for c in (1, 2, 4, 8, 16) if mcol_tile_ok(L, c)]
    assert widths
    for ct in widths:
        cols, rows, nt = column_partials(L, M, 1, ct, False)
        assert nt == ct * L // 16 and nt % ct == 0
        assert len(cols) == gcols and np.array_equal(np.sort(cols), np.arange(gcols))
        for (b, tc), rr in rows.items():
            assert rr == [tc + j * (L // 16) for j in range(16)]
