"""The box-grid kernel's schedule (raptor_b200/csrc/grid.cuh, k_grid_rows)
restated on the CPU, over box sizes that are not multiples of its tiles or
of its planes per block, for every stencil shape and one or two rows in x a
thread.  Mirroring the kernel's index arithmetic block by block (flattened
block index, x fastest; the per-thread plane loads; the four-buffer ring and
its z loop unrolled by four), it checks what the kernel relies on: every
global load lies inside x, every shared-memory read inside its plane buffer
(and, with two rows a thread, on an even index, so that the pair loads are
aligned), every row is written exactly once, and the result is the
zero-padded stencil product.
"""
import numpy as np
import pytest


def shape(s):
    if s == "box27":
        return [(d // 9 - 1, (d // 3) % 3 - 1, d % 3 - 1) for d in range(27)], 1
    if s == "star7":
        return [(-1, 0, 0), (0, -1, 0), (0, 0, -1), (0, 0, 0), (0, 0, 1), (0, 1, 0), (1, 0, 0)], 1
    if s == "box9":
        return [(d // 3 - 1, 0, d % 3 - 1) for d in range(9)], 0
    return [(-1, 0, 0), (0, 0, -1), (0, 0, 0), (0, 0, 1), (1, 0, 0)], 0


def run_schedule(s, vx, nx, ny, nz, zc):
    sh, hy = shape(s)
    txt = 32 if hy else 256
    txw, tyh = txt * vx, (8 if hy else 1)
    W, H = txw + 2, tyh + 2 * hy
    P, NT = W * H, txt * tyh
    lpt = (P + NT - 1) // NT
    assert W % 2 == 0 and P % 2 == 0
    n = nx * ny * nz
    rng = np.random.default_rng(1)
    x = rng.standard_normal(n)
    c = rng.standard_normal(len(sh))
    y = np.full(n, np.nan)
    cnt = np.zeros(n, int)
    ntx, nty = -(-nx // txw), -(-ny // tyh)
    t = np.arange(NT)
    for blk in range(ntx * nty * -(-nz // zc)):
        bx, bt = blk % ntx, blk // ntx
        by, bz = bt % nty, bt // nty
        x0, y0, z0 = bx * txw, by * tyh, bz * zc
        tx, ty = t % txt, t // txt
        goff, gok, es = [], [], []
        for u in range(lpt):
            e = t + u * NT
            gy, gx = y0 - hy + e // W, x0 - 1 + e % W
            gok.append((e < P) & (gy >= 0) & (gy < ny) & (gx >= 0) & (gx < nx))
            goff.append(gy * nx + gx)
            es.append(e)
        buf = np.full((4, P), np.nan)

        def load(zp):
            v = []
            for u in range(lpt):
                vv = np.zeros(NT)
                m = gok[u] & (0 <= zp < nz)
                idx = zp * nx * ny + goff[u][m]
                assert np.all((idx >= 0) & (idx < n))
                vv[m] = x[idx]
                v.append(vv)
            return v

        def store(slot, v):
            for u in range(lpt):
                m = es[u] < P if u == lpt - 1 else np.ones(NT, bool)
                buf[slot, es[u][m]] = v[u][m]

        for k, zp in enumerate((z0 - 1, z0, z0 + 1)):
            store(k, load(zp))
        zend = min(z0 + zc, nz)
        left = (ty + hy) * W + tx * vx
        xr = x0 + tx * vx
        inr = [(y0 + ty < ny) & (xr + r < nx) for r in range(vx)]
        rowxy = (y0 + ty) * nx + xr
        for z in range(z0, zend, 4):
            for K in range(4):
                zz = z + K
                if zz >= zend:
                    break
                more = zz + 1 < zend
                if more:
                    v = load(zz + 2)
                acc = [np.zeros(NT) for _ in range(vx)]
                for d, (dz, dy, dx) in enumerate(sh):
                    row = left + dy * W
                    slot = (K + 1 + dz) & 3
                    if vx == 1:
                        idx = row + 1 + dx
                        assert np.all((idx >= 0) & (idx < P))
                        acc[0] = acc[0] + c[d] * buf[slot, idx]
                    else:
                        assert np.all(row % 2 == 0) and np.all(row >= 0)
                        assert np.all(row % W + 3 < W) and np.all(row + 3 < P)
                        vals = [buf[slot, row + q] for q in range(4)]
                        acc[0] = acc[0] + c[d] * vals[1 + dx]
                        acc[1] = acc[1] + c[d] * vals[2 + dx]
                i = zz * nx * ny + rowxy
                for r in range(vx):
                    ii = (i + r)[inr[r]]
                    assert np.all(ii < n)
                    y[ii] = acc[r][inr[r]]
                    cnt[ii] += 1
                if more:
                    store((K + 3) & 3, v)
    assert np.all(cnt == 1)
    X = np.pad(x.reshape(nz, ny, nx), 1)
    ref = np.zeros((nz, ny, nx))
    for d, (dz, dy, dx) in enumerate(sh):
        ref += c[d] * X[1 + dz:1 + dz + nz, 1 + dy:1 + dy + ny, 1 + dx:1 + dx + nx]
    np.testing.assert_allclose(y, ref.ravel(), rtol=0, atol=1e-12)


CASES = [("box27", 37, 19, 23, 8), ("box27", 3, 3, 5, 32), ("box27", 3, 3, 1, 8),
         ("box27", 65, 16, 9, 5), ("box27", 130, 9, 4, 16), ("star7", 40, 9, 13, 8),
         ("star7", 33, 3, 7, 6), ("box9", 500, 1, 37, 12), ("box9", 513, 1, 3, 4),
         ("star5", 257, 1, 11, 24)]


@pytest.mark.parametrize("vx", [1, 2])
@pytest.mark.parametrize("case", CASES, ids=lambda c: "%s_%dx%dx%d_zc%d" % c)
def test_grid_schedule(case, vx):
    s, nx, ny, nz, zc = case
    run_schedule(s, vx, nx, ny, nz, zc)
