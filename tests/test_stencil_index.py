"""CPU checks of the stencil kernels' neighbour addressing against the oracle's layout
(the 3D Laplacian kernels; the batch residual step's in-block offsets at the end).

``stencil3d_lines_kernel`` (stencilfft_b200/csrc/zm_stencil.cu) finds the y / z
neighbour lines through the block-cyclic maps and the x neighbours across a block edge
through a closed form (rank +-1, or -+(P - 1) with a one-element shift past the end of a
block cycle).  This restates that integer arithmetic in numpy and checks every neighbour
of every element against the real-layout permutation of the oracle (zoracle.c, the
reference's utils.h index maps): the element at natural (d, r, c +- 1) etc.  It also
checks that the warp / lane / vector assignment covers every vector once.  The kernel's
own outputs are checked against the oracle by the GPU parity tests.
"""
import numpy as np
import pytest

import oracle as O


def lg(x):
    return int(x).bit_length() - 1


def kernel_neighbours(n, b, p, K):
    """Element index of each neighbour of each element, as the kernel computes it:
    returns {name: array over all elements e of the real layout}."""
    L = n // p
    vec = L // b
    logB, logP, logL, logVEC = lg(b), lg(p), lg(L), lg(vec)
    total = L ** 3 * p ** 3
    e = np.arange(total, dtype=np.int64)
    line, pos_e = e >> logL, e & (L - 1)
    k = pos_e & (K - 1)                  # element inside its 16-byte vector
    pos = pos_e - k                      # the vector's first packed position
    lr, ld, rank = line & (L - 1), (line >> logL) & (L - 1), line >> (2 * logL)
    cid, rid, did = rank & (p - 1), (rank >> logP) & (p - 1), rank >> (2 * logP)

    def l2g(li, i):
        return ((li >> logB) << (logB + logP)) + (i << logB) + (li & (b - 1))

    def g2l(gi):
        return (gi >> logB) & (p - 1), ((gi >> (logB + logP)) << logB) + (gi & (b - 1))

    gr, gd = l2g(lr, rid), l2g(ld, did)
    ec = line << logL
    out = {}
    for d, nm in ((-1, "up"), (1, "dn")):
        i, li = g2l((gr + d + n) & (n - 1))
        rk = (did * p + i) * p + cid
        out[nm] = (((((rk << logL) + ld) << logL) + li) << logL) + pos + k
    for d, nm in ((-1, "fr"), (1, "bk")):
        i, li = g2l((gd + d + n) & (n - 1))
        rk = (i * p + rid) * p + cid
        out[nm] = (((((rk << logL) + li) << logL) + lr) << logL) + pos + k
    l3 = L ** 3
    j, jj = pos >> logVEC, pos & (vec - 1)
    for d, nm in ((-1, "lf"), (1, "rt")):
        inside = j > 0 if d < 0 else j < b - 1
        wrap = cid == 0 if d < 0 else cid == p - 1
        e1 = ec + np.where(wrap, -d * (p - 1), d) * l3 + ((b - 1) << logVEC if d < 0 else 0)
        edge = np.where(wrap, e1 + ((jj + k + d) & (vec - 1)), e1 + jj + k)
        out[nm] = np.where(inside, ec + pos + k + d * vec, edge)
    return out


def true_neighbours(n, b, p):
    fwd = O.real_layout_map(3, n, b, p)          # real element -> natural index
    inv = O.real_layout_inverse_map(3, n, b, p)  # natural index -> real element
    d, r, c = fwd // (n * n), (fwd // n) % n, fwd % n
    nat = lambda dd, rr, cc: ((dd % n) * n + rr % n) * n + cc % n
    return {"up": inv[nat(d, r - 1, c)], "dn": inv[nat(d, r + 1, c)],
            "lf": inv[nat(d, r, c - 1)], "rt": inv[nat(d, r, c + 1)],
            "fr": inv[nat(d - 1, r, c)], "bk": inv[nat(d + 1, r, c)]}


# (N, B, P) with P dividing VEC = N / (P B); P = 1, 2, 4, 8 and VEC from 1 to 8
CONFIGS = [(16, 2, 2), (32, 2, 4), (32, 4, 2), (64, 4, 4), (64, 8, 2), (64, 16, 2),
           (128, 2, 8), (16, 16, 1), (32, 8, 1)]


@pytest.mark.parametrize("n,b,p", CONFIGS)
@pytest.mark.parametrize("K", [1, 2])
def test_laplace3d_neighbours_match_layout(n, b, p, K):
    vec = n // p // b
    if vec % K:
        pytest.skip("the kernel needs VEC to be a multiple of the elements per vector")
    got, ref = kernel_neighbours(n, b, p, K), true_neighbours(n, b, p)
    for nm in ref:
        assert np.array_equal(got[nm], ref[nm]), nm


@pytest.mark.parametrize("L,K,RX", [(64, 1, 2), (128, 1, 4), (128, 2, 2), (256, 2, 2)])
def test_laplace3d_warp_assignment_covers_each_vector_once(L, K, RX):
    lines = 64                           # any count: the map is per line
    nvec = lines * L // K
    nseg = nvec // (32 * RX)
    segs_line = L // (K * 32 * RX)
    tid = np.arange(nseg * 32, dtype=np.int64)
    seg, lane = tid >> 5, tid & 31
    line = seg // segs_line
    v0 = (seg - line * segs_line) * 32 * RX + lane
    first = np.concatenate([line * L + (v0 + 32 * x) * K for x in range(RX)])
    assert np.array_equal(np.sort(first), np.arange(0, lines * L, K))
    # each warp instruction reads 32 consecutive vectors of one line
    for x in range(RX):
        pos = (v0 + 32 * x) * K
        w = pos.reshape(-1, 32)
        assert (np.diff(w, axis=1) == K).all() and (w[:, -1] < L).all()


@pytest.mark.parametrize("n,b,p", CONFIGS)
def test_laplace3d_global_line_order_is_a_permutation(n, b, p):
    """The complex128 form of the kernel walks lines in global order (global depth, global
    row, then the P ranks of that row): the map from that order to (rank * L + ld) * L + lr
    visits every line of every rank once."""
    L = n // p
    logB, logP, logL, logN = lg(b), lg(p), lg(L), lg(n)
    gline = np.arange(p * n * n, dtype=np.int64)
    cid = gline & (p - 1)
    gr, gd = (gline >> logP) & (n - 1), gline >> (logP + logN)

    def g2l(gi):
        return (gi >> logB) & (p - 1), ((gi >> (logB + logP)) << logB) + (gi & (b - 1))

    rid, lr = g2l(gr)
    did, ld = g2l(gd)
    rank = (did * p + rid) * p + cid
    line = (((rank << logL) + ld) << logL) + lr
    assert np.array_equal(np.sort(line), np.arange(p ** 3 * L * L))


def march_neighbours(n, b, p, ty, zsteps):
    """Element index of each neighbour of each element as stencil3d_march_kernel reads it:
    a CTA owns local rows lr0 .. lr0 + ty - 1 of rank column (rid, cid) and walks a chunk
    of zsteps global depths, upwards in even chunks and downwards in odd ones; walk step k
    fills slot k mod 4 with rows [halo above, ty rows, halo below] of the rank of its depth
    (halos through the block-cyclic row maps) and, for centre planes, an edge area with the
    last vector of the left rank's row and the first vector of the right rank's row per
    tile row; y / z neighbours come from the slots, x neighbours from the slot row or,
    across a block edge, from the edge area (shifted by one element at the periodic wrap)."""
    L = n // p
    vec = L // b
    logB, logP, logL, logVEC = lg(b), lg(p), lg(L), lg(vec)

    def l2g(li, i):
        return ((li >> logB) << (logB + logP)) + (i << logB) + (li & (b - 1))

    def g2l(gi):
        return (gi >> logB) & (p - 1), ((gi >> (logB + logP)) << logB) + (gi & (b - 1))

    def row_elem(rk, ld, lr):
        return ((rk * L + ld) * L + lr) * L

    total = L ** 3 * p ** 3
    out = {k: np.full(total, -1, dtype=np.int64) for k in ("up", "dn", "lf", "rt", "fr", "bk")}
    l3 = L ** 3
    pos = np.arange(L)
    j, jj = pos >> logVEC, pos & (vec - 1)
    for rid in range(p):
        for cid in range(p):
            dl = (p - 1) * l3 if cid == 0 else -l3
            dr = -(p - 1) * l3 if cid == p - 1 else l3
            shl = -1 if cid == 0 else 0
            shr = 1 if cid == p - 1 else 0
            for lr0 in range(0, L, ty):
                ridU, lrU = g2l((l2g(lr0, rid) - 1 + n) % n)
                ridD, lrD = g2l((l2g(lr0 + ty - 1, rid) + 1) % n)
                for zc in range(n // zsteps):
                    gd0, down = zc * zsteps, zc % 2 == 1

                    def depth(k):
                        return gd0 + zsteps - k if down else gd0 - 1 + k

                    def slot(k):   # (rows, left edge vectors, right edge vectors)
                        did, ld = g2l(depth(k) % n)
                        rk = (did * p + rid) * p + cid
                        rows = [row_elem((did * p + ridU) * p + cid, ld, lrU)]
                        rows += [row_elem(rk, ld, lr0 + r) for r in range(ty)]
                        rows += [row_elem((did * p + ridD) * p + cid, ld, lrD)]
                        eb = row_elem(rk, ld, lr0)
                        el = [eb + r * L + dl + (b - 1) * vec + np.arange(vec) for r in range(ty)]
                        er = [eb + r * L + dr + np.arange(vec) for r in range(ty)]
                        return rows, el, er
                    for z in range(zsteps):
                        s0, sc, s2 = slot(z), slot(z + 1), slot(z + 2)
                        sm, sp = (s2, s0) if down else (s0, s2)
                        for r in range(ty):
                            ec = sc[0][r + 1]
                            e = ec + pos
                            out["up"][e] = sc[0][r] + pos
                            out["dn"][e] = sc[0][r + 2] + pos
                            out["fr"][e] = sm[0][r + 1] + pos
                            out["bk"][e] = sp[0][r + 1] + pos
                            out["lf"][e] = np.where(j > 0, ec + pos - vec, sc[1][r][(jj + shl) & (vec - 1)])
                            out["rt"][e] = np.where(j < b - 1, ec + pos + vec, sc[2][r][(jj + shr) & (vec - 1)])
    return out


@pytest.mark.parametrize("n,b,p", [(16, 4, 2), (32, 4, 2), (64, 4, 4), (64, 8, 2), (64, 16, 2), (32, 8, 1)])
def test_laplace3d_plane_tiles_match_layout(n, b, p):
    """The plane-tile kernel's neighbour addressing equals the true neighbours for every
    element (tile heights as the launcher picks them: min(8, B) for complex64 and
    min(4, B) for complex128; one chunk of all depths, and chunks of 8 walked in
    alternating directions)."""
    ref = true_neighbours(n, b, p)
    for ty in sorted({min(8, b), min(4, b)}):
        if ty < 2 or (n // p) % ty:
            continue
        for zsteps in sorted({n, 8}):
            got = march_neighbours(n, b, p, ty, zsteps)
            for nm in ref:
                assert (got[nm] >= 0).all(), (nm, ty, zsteps)
                assert np.array_equal(got[nm], ref[nm]), (nm, ty, zsteps)


@pytest.mark.parametrize("n,b,p", [(32, 4, 2), (64, 4, 2), (64, 8, 2), (128, 8, 4), (128, 16, 2), (256, 32, 2),
                                   (64, 16, 2), (128, 4, 4)])
def test_batch_residual_interior_offsets_match_layout(n, b, p):
    """The batch residual step (zm_batch.cu, residual_tile) takes the four neighbours of an
    element pair (e, e + 1), e even, at e -+ L (rows) and e -+ VEC (columns) when the pair
    lies inside its rank's B x B block (in-block column j = pos >> log VEC and row lr mod B
    both off the block's edges) and VEC >= 2.  Check every such pair against the true
    neighbours of the 2D real layout (the oracle's restatement of utils.h), and that the
    pair shares its in-block column."""
    L = n // p
    vec = L // b
    fwd = O.real_layout_map(2, n, b, p)
    inv = O.real_layout_inverse_map(2, n, b, p)
    r, c = fwd // n, fwd % n
    nat = lambda rr, cc: (rr % n) * n + cc % n
    true = {"up": inv[nat(r - 1, c)], "dn": inv[nat(r + 1, c)], "lf": inv[nat(r, c - 1)], "rt": inv[nat(r, c + 1)]}
    e = np.arange(0, L * L * p * p, 2, dtype=np.int64)
    pos, lr = e & (L - 1), (e >> lg(L)) & (L - 1)
    j, rb = pos >> lg(vec), lr & (b - 1)
    fast = (vec >= 2) & (j > 0) & (j < b - 1) & (rb > 0) & (rb < b - 1)
    if vec >= 2:
        assert fast.any()
    assert np.array_equal((pos + 1) >> lg(vec), j)          # e + 1 in the same in-block column
    for k in (0, 1):
        ee = e[fast] + k
        assert np.array_equal(true["up"][ee], ee - L)
        assert np.array_equal(true["dn"][ee], ee + L)
        assert np.array_equal(true["lf"][ee], ee - vec)
        assert np.array_equal(true["rt"][ee], ee + vec)
