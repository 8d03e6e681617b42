"""The arithmetic of the fused projector pair (csrc/zpath.cuh), restated in
numpy and checked on the CPU:

* the convolution passes over zero-padded lines whose data start at
  D0 = h rounded up to 4, with the weights shifted right by D0 - h and the
  clamped boundary added as tail terms (forward) or folded (adjoint), equal the
  replicate-boundary convolution of fft_conv! and its adjoint
  (src/fft_convolve.jl:33-130) -- against the oracle's FFT convolution;
* the gather form of imrotate_adj! :two (src/rotatez.jl:390-416): the
  rotated-grid points whose bilinear footprint covers an output pixel are all
  within |cos| + |sin| of the inverse-rotated pixel (at most 3 x 3
  candidates), so the gather is the exact transpose of the forward sampling
  computed with the forward's float32 operations;
* the buffer geometry of the kernels (zgeom_make): every shared-memory and
  global index the kernels form stays inside its buffer, for a sweep of sizes.
"""
import numpy as np
import pytest

from conftest import relerr

F = np.float32


def zround(v, m):
    return (v + m - 1) // m * m


def zstride4(v):
    r = zround(v, 4)
    return r if (r // 4) % 2 == 1 else r + 4


def zgeom(nx, nz, px, pz):
    """Python mirror of zgeom_make (csrc/zpath_api.h)."""
    pad = int(np.ceil(1.0 + nx * np.sqrt(2.0) / 2.0 - nx / 2.0))
    g = dict(nx=nx, ny=nx, nz=nz, nzp=zround(nz, 16), pad=pad, L=nx + 2 * pad, px=px, pz=pz,
             hx=(px - 1) // 2, hz=(pz - 1) // 2)
    g["R0"], g["C0"] = zround(g["hz"], 4), zround(g["hx"], 4)
    g["zpw"] = zround(g["R0"] - g["hz"] + pz, 8)
    g["xpw"] = zround(g["C0"] - g["hx"] + px, 8)
    g["hs"] = g["zpw"] + g["xpw"]
    g["ts"] = max(4, zround(2 * g["hx"] + 2 * g["hz"], 4))
    g["rows"] = zround(nz, 16) + g["zpw"]
    g["ast"] = zstride4(g["rows"])
    g["bs"] = zstride4(nx + g["xpw"])
    return g


def gauss(p, sigma):
    x = np.arange(p) - (p - 1) // 2
    g = np.exp(-x * x / (2.0 * sigma * sigma))
    return g / g.sum()


def clamp_conv(line, w):
    """Reference: out[i] = sum_d w(d) line[clamp(i - d)] for the centred factor w."""
    n, p = line.shape[0], w.shape[0]
    h = (p - 1) // 2
    return np.array([sum(w[d + h] * line[min(max(i - d, 0), n - 1)] for d in range(-h, h + 1)) for i in range(n)])


def fused_fwd_pass(line, w):
    """The kernels' forward pass: 8-output tasks over the zero-padded buffer
    (data at D0), shifted reversed weights, clamp tails EL/ER."""
    n, p = line.shape[0], w.shape[0]
    h = (p - 1) // 2
    D0 = zround(h, 4)
    sh = D0 - h
    win = zround(sh + p, 8)
    rows = zround(n, 8) + win
    buf = np.zeros(rows + 8)
    buf[D0:D0 + n] = line
    ws = np.zeros(win)
    ws[sh:sh + p] = w[::-1]
    wr = w[::-1]
    EL = [wr[:h - i].sum() for i in range(h)]
    ER = [wr[h + 1 + k:].sum() for k in range(h)]
    out = np.zeros(zround(n, 8))
    for z0 in range(0, zround(n, 8), 8):
        for k in range(8):
            i = z0 + k
            out[i] = sum(ws[m] * buf[i + m] for m in range(win))
            if i < h:
                out[i] += EL[i] * buf[D0]
            kk = n - 1 - i
            if 0 <= kk < h:
                out[i] += ER[kk] * buf[D0 + n - 1]
    return out[:n]


def fused_adj_pass(u, w):
    """The kernels' adjoint pass: zero-padded correlation with the shifted
    factor, folds cL/cR at the two ends."""
    n, p = u.shape[0], w.shape[0]
    h = (p - 1) // 2
    D0 = zround(h, 4)
    sh = D0 - h
    win = zround(sh + p, 8)
    buf = np.zeros(zround(n, 8) + win + 8)
    buf[D0:D0 + n] = u
    ws = np.zeros(win)
    ws[sh:sh + p] = w
    cl = [w[h + k + 1:].sum() for k in range(h)]
    cr = [w[:h - k].sum() for k in range(h)]
    out = np.array([sum(ws[m] * buf[i + m] for m in range(win)) for i in range(n)])
    out[0] += sum(cl[k] * buf[D0 + k] for k in range(h))
    out[n - 1] += sum(cr[k] * buf[D0 + n - 1 - k] for k in range(h))
    return out


@pytest.mark.parametrize("n,p", [(80, 37), (64, 11), (128, 21), (12, 37), (1, 1), (8, 3), (200, 65), (5, 9)])
def test_fused_passes_equal_clamped_convolution(n, p):
    rng = np.random.default_rng(n * 100 + p)
    w = gauss(p, 1.0 + p / 8.0)
    line = rng.random(n)
    assert relerr(fused_fwd_pass(line, w), clamp_conv(line, w)) < 1e-12
    # adjoint: <C x, u> == <x, C' u>
    u = rng.random(n)
    lhs = float(np.dot(clamp_conv(line, w), u))
    rhs = float(np.dot(line, fused_adj_pass(u, w)))
    assert abs(lhs - rhs) <= 1e-12 * abs(lhs)


def test_fused_plane_against_oracle_fft_conv():
    """A full plane: z pass then x pass (forward) and the two adjoint passes,
    against the oracle's fft_conv!/fft_conv_adj! of the rank-1 kernel."""
    from oracle import oracle as O

    rng = np.random.default_rng(5)
    nx, nz, px, pz = 40, 24, 13, 9
    a, b = gauss(px, 2.0), gauss(pz, 1.5)
    img = rng.random((nx, nz))
    ker = np.outer(a, b)
    zp = np.stack([fused_fwd_pass(img[i, :], b) for i in range(nx)])
    out = np.stack([fused_fwd_pass(zp[:, j], a) for j in range(nz)], axis=1)
    ref = O.fft_conv(img, ker, dtype=np.float64)
    assert relerr(out, ref) < 1e-12
    xa = np.stack([fused_adj_pass(img[:, j], a) for j in range(nz)], axis=1)
    adj = np.stack([fused_adj_pass(xa[i, :], b) for i in range(nx)])
    refa = O.fft_conv(img, ker, adj=True, dtype=np.float64)
    assert relerr(adj, refa) < 1e-12


def fwd_taps(nx, cs, sn):
    """The forward sampling with float32 operations in the kernels' order:
    for every rotated-grid point (x, y) its lower-left tap (f1, f2) and
    (t1, t2), as arrays over (y, x)."""
    c0 = F((nx - 1) * 0.5)
    o = np.arange(nx, dtype=F)
    di = (o - c0).astype(F)
    a = (F(cs) * di)[None, :]
    c = (F(sn) * di)[None, :]
    b = (F(sn) * di)[:, None]
    d = (F(cs) * di)[:, None]
    s1 = (c0 + (a - b)).astype(F)
    s2 = (c0 + (c + d)).astype(F)
    return s1, s2


@pytest.mark.parametrize("nx,nview", [(128, 120), (64, 64), (16, 6), (96, 90)])
def test_gather_candidates_cover_the_forward_footprints(nx, nview):
    """For every view angle: each rotated-grid point's four taps are found by
    the gather's candidate box around the inverse-rotated pixel, and nothing
    else passes the gather's range test."""
    c0 = (nx - 1) * 0.5
    for v in range(nview):
        theta = np.float32(v / nview * np.float32(2 * np.pi))
        phi = 2 * np.pi - float(theta)
        cs, sn = F(np.cos(phi)), F(np.sin(phi))
        s1, s2 = fwd_taps(nx, cs, sn)
        f1, f2 = np.floor(s1).astype(int), np.floor(s2).astype(int)
        yy, xx = np.meshgrid(np.arange(nx), np.arange(nx), indexing="ij")
        # forward: pixel -> set of contributing points
        want = {}
        for ty in (0, 1):
            for tx in (0, 1):
                j1, j2 = f1 + tx, f2 + ty
                ok = (j1 >= 0) & (j1 < nx) & (j2 >= 0) & (j2 < nx)
                for p_, x_, y_ in zip((j2 * nx + j1)[ok], xx[ok], yy[ok]):
                    want.setdefault(int(p_), set()).add((int(x_), int(y_)))
        # gather: candidates within |cos| + |sin| + 0.01 of the inverse centre
        rr = float(F(abs(float(cs)) + abs(float(sn)) + 0.01))
        for p_, pts in want.items():
            j2, j1 = divmod(p_, nx)
            d1, d2 = j1 - c0, j2 - c0
            xc = c0 + float(cs) * d1 + float(sn) * d2
            yc = c0 - float(sn) * d1 + float(cs) * d2
            xs = range(max(0, int(np.ceil(xc - rr))), min(nx - 1, int(np.floor(xc + rr))) + 1)
            ys = range(max(0, int(np.ceil(yc - rr))), min(nx - 1, int(np.floor(yc + rr))) + 1)
            assert len(xs) <= 3 and len(ys) <= 3
            got = {(x_, y_) for x_ in xs for y_ in ys
                   if j1 - 1 <= s1[y_, x_] < j1 + 1 and j2 - 1 <= s2[y_, x_] < j2 + 1}
            assert got == pts, (v, p_, got ^ pts)


@pytest.mark.parametrize("nx,nz,px,pz", [(128, 80, 37, 37), (64, 64, 11, 11), (96, 48, 21, 21), (128, 128, 37, 37),
                                         (16, 12, 5, 3), (64, 1, 11, 1), (256, 200, 65, 65), (64, 90, 21, 21)])
def test_fused_buffer_bounds(nx, nz, px, pz):
    """Every index the fused kernels form stays inside its buffer."""
    g = zgeom(nx, nz, px, pz)
    nz4 = (nz + 3) // 4
    assert g["ast"] % 4 == 0 and (g["ast"] // 4) % 2 == 1 and g["bs"] % 4 == 0 and (g["bs"] // 4) % 2 == 1
    assert g["hs"] % 8 == 0 and g["ts"] % 4 == 0 and g["nzp"] % 16 == 0
    # z-pass buffer: build stores rows R0 + 4 zg + 3
    assert g["R0"] + 4 * nz4 <= g["ast"]
    assert g["R0"] + nz <= g["ast"]  # adjoint x-pass stores and edge reads
    for W in (8, 16):  # task widths; W = 16 only where W divides nx
        nzb = (nz + W - 1) // W
        # windows read rows z0 .. z0 + zpw + W - 1; adjoint z-pass stores z0 .. z0 + W - 1 of a T column
        assert W * (nzb - 1) + g["zpw"] + W <= g["rows"] <= g["ast"]
        assert W * nzb <= g["nzp"]
        if nx % W:
            continue
        # x-pass buffer: z-pass stores column C0 + nx - 1; windows read x0 .. x0 + xpw + W - 1
        assert g["C0"] + nx <= g["bs"] and (nx - W) + g["xpw"] + W <= g["bs"]
    # tap shift inside the window
    assert g["R0"] - g["hz"] + pz <= g["zpw"] and g["C0"] - g["hx"] + px <= g["xpw"]
    # IZ: the farthest tap of the farthest in-grid sample, plus the z group
    L, nzp = g["L"], g["nzp"]
    jmax = nx + g["pad"] - 2
    top = ((jmax + g["pad"]) * L + jmax + g["pad"]) * nzp + L * nzp + nzp + 4 * nz4 - 1
    assert top < L * L * nzp
    # every sample of the cropped grid lies inside the padded grid
    r = (nx - 1) / 2 * np.sqrt(2.0)
    assert np.floor((nx - 1) / 2 - r) >= -g["pad"] and np.floor((nx - 1) / 2 + r) <= jmax
    # the adjoint planes' z blocks end inside the padded column
    assert 8 * nzb <= nzp


def trim_taps(w):
    """Mirror of trim_taps (csrc/spect_gpu.cu): zero the outer taps while their
    summed magnitude per side stays within 2^-27 of the factor's."""
    w = np.array(w, np.float64)
    lim = np.ldexp(np.abs(w).sum(), -27)
    acc = 0.0
    for i in range(len(w)):
        acc += abs(w[i])
        if acc > lim:
            break
        w[i] = 0.0
    acc = 0.0
    for i in range(len(w) - 1, -1, -1):
        acc += abs(w[i])
        if acc > lim:
            break
        w[i] = 0.0
    return w


def tap_range(row):
    """Mirror of tap_range: (first 4-tap block, 8-tap blocks) covering the
    nonzero taps of a pass row, within the row."""
    nzi = np.flatnonzero(row)
    lo, hi = nzi[0], nzi[-1]
    b = lo // 4
    n = (hi + 1 - 4 * b + 7) // 8
    if 4 * b + 8 * n > len(row):
        b -= 1
    return b, n


@pytest.mark.parametrize("nx,nz,p,f0,f1", [(128, 80, 37, 1.0, 6.0), (64, 64, 11, 1.0, 3.0), (256, 200, 65, 1.0, 6.0),
                                          (96, 48, 21, 0.5, 8.0), (40, 37, 9, 1.0, 2.5)])
def test_trimmed_taps_and_ranges(nx, nz, p, f0, f1):
    """Trimmed factors leave out at most 2^-26 of a factor's mass; each pass's
    tap-block range covers every kept tap and stays inside its row; the
    trimmed clamped convolution equals the full one to 2^-24 relative."""
    from oracle import oracle as O
    g = zgeom(nx, nz, p, p)
    psf = O.psf_gauss(nx, p, p, f0, f1, None, None, None, np.float64)
    h = (p - 1) // 2
    rng = np.random.default_rng(p)
    line = rng.random(nz)
    for y in range(0, nx, max(1, nx // 16)):
        a = psf[:, h, y] / psf[h, h, y]
        t = trim_taps(a)
        assert np.abs(a - t).sum() <= 2.0 ** -26 * np.abs(a).sum()
        assert t[h] == a[h]
        s = g["R0"] - g["hz"]
        row = np.zeros(g["zpw"])
        row[s:s + p] = t[::-1]
        b4, n8 = tap_range(row)
        assert b4 >= 0 and n8 >= 1 and 4 * b4 + 8 * n8 <= g["zpw"]
        nzi = np.flatnonzero(row)
        assert 4 * b4 <= nzi[0] and nzi[-1] < 4 * b4 + 8 * n8
        full, cut = clamp_conv(line, a[::-1]), clamp_conv(line, t[::-1])
        assert np.abs(full - cut).max() <= 2.0 ** -24 * np.abs(full).max()


def zs_tiles(g, optin=232448):
    """Mirror of zs_tiles (csrc/spect_gpu.cu): task width, column tile, row tile."""
    nx, nz = g["nx"], g["nz"]
    w = 16 if nx % 16 == 0 else 8
    tx = 32 if nx % 32 == 0 else (16 if nx % 16 == 0 else 8)
    tz = min(640 * w // nx // 4 * 4, zround(nz, 4))
    hts = g["hs"] + g["ts"] + 4
    smem = {"fz": 4 * (hts + 5 * tx + tx * g["ast"] + nz * tx),
            "fx": 4 * 2 * (tz * g["bs"] + hts),
            "adj": 4 * (nz * zstride4(tx + g["xpw"]) + tx * g["ast"] + hts)}
    return w, tx, tz, smem


@pytest.mark.parametrize("nx,nz,px,pz", [(256, 200, 65, 65), (128, 80, 37, 37), (128, 128, 37, 37), (512, 96, 21, 21),
                                         (64, 37, 9, 9), (96, 48, 21, 21)])
def test_large_plane_tile_bounds(nx, nz, px, pz):
    """Every index the large-plane kernels form stays inside its buffer, and
    their shared memory fits at the benchmark's large study."""
    g = zgeom(nx, nz, px, pz)
    w, tx, tz, smem = zs_tiles(g)
    assert tz >= 4 and tz % 4 == 0 and nx % tx == 0 and tx % 4 == 0 and nx % w == 0
    # k_zs_fx: one x task per thread, the prefetch holds a plane's rows in four float4 a thread
    assert tz * (nx // w) <= 640 and tz * nx // 4 <= 4 * 640
    # its rows: data at C0 .. C0 + nx - 1, windows read x0 .. x0 + xpw + w - 1
    assert g["C0"] + nx <= g["bs"] and (nx - w) + g["xpw"] + w <= g["bs"]
    # k_zs_fz / k_zs_adj z pass: column rows as the fused kernels (R0 + 4 nz4 <= ast, windows <= rows)
    nzb = (nz + w - 1) // w
    assert g["R0"] + 4 * ((nz + 3) // 4) <= g["ast"] and w * (nzb - 1) + g["zpw"] + w <= g["rows"] <= g["ast"]
    # k_zs_adj tile lines: windows read x0 .. x0 + xpw + w - 1 (x0 <= tx - w); the left fold
    # (first tile, x0 = 0) reads C0 .. C0 + hx - 1, the right fold (last tile, x0 = tx - w)
    # C0 + tx - hx .. C0 + tx - 1
    tbs = zstride4(tx + g["xpw"])
    assert (tx - w) + g["xpw"] + w <= tbs and g["C0"] + g["hx"] <= tbs
    assert g["C0"] + tx - g["hx"] >= 0 and g["C0"] + tx - 1 < tbs
    if (nx, nz, px) == (256, 200, 65):
        assert max(smem.values()) <= 232448, smem
