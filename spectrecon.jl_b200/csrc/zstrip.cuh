// zstrip.cuh -- the projector pair for planes too large for the fused
// kernels' shared memory (e.g. 256x256x200 with a 65-tap PSF), on the same
// z-fastest layouts (IZ image, ATT cache, T adjoint planes) and with the same
// trimmed separable passes (zpassw, tail and fold tables, tap ranges) as
// zpath.cuh, over plane tiles; the forward's two passes are kernels of their
// own that exchange planes through the device buffer Q.
//
// forward (project!, src/project.jl:77-135):
//   k_zs_fz  item (slot, y, tile of tx columns): gather the rotated,
//            attenuated columns (as k_zfwd), z pass, rows -> Q[slot][y][z][x]
//   k_zs_fx  item (slot, depth chunk, tile of tz rows): per plane the rows of
//            Q (loaded one plane ahead into registers), x pass accumulated
//            over the chunk -> part[slot][chunk][z][x]
// adjoint (backproject!, src/backproject.jl:69-124), convolution half:
//   k_zs_adj item (slot, tile of tx columns, depth chunk): the view's columns
//            of the tile and its halo once; per plane the x pass, the z pass
//            times the attenuation -> T[slot][y][x][nzp]
// Every output goes through the operations of the fused kernels in the same
// order (z then x in the forward, x then z in the adjoint), so the two paths
// agree bit for bit.
#pragma once
#include "zpath.cuh"

namespace spect {

// the sample geometry of column x of plane y for the view's (cos, sin):
// k_zfwd's geometry, one column
__device__ __forceinline__ void zs_geometry(const ZGeom& g, float4 r, int x, int y, float4* w_out, int* o_out) {
  int j1 = x, j2 = y;
  float4 w = make_float4(1.f, 0.f, 0.f, 0.f);
  if (r.z == 0.f) {
    const float cs = r.x, sn = r.y;
    const float d1 = __fsub_rn((float)x, g.c0), d2 = __fsub_rn((float)y, g.c0);
    const float s1 = __fadd_rn(g.c0, __fsub_rn(__fmul_rn(cs, d1), __fmul_rn(sn, d2)));
    const float s2 = __fadd_rn(g.c0, __fadd_rn(__fmul_rn(sn, d1), __fmul_rn(cs, d2)));
    const float f1 = floorf(s1), f2 = floorf(s2);
    const float t1 = __fsub_rn(s1, f1), t2 = __fsub_rn(s2, f2);
    const float u1 = __fsub_rn(1.0f, t1), u2 = __fsub_rn(1.0f, t2);
    j1 = (int)f1;
    j2 = (int)f2;
    w = make_float4(__fmul_rn(u1, u2), __fmul_rn(t1, u2), __fmul_rn(u1, t2), __fmul_rn(t1, t2));
    if (j1 < -g.pad || j1 > g.nx + g.pad - 2 || j2 < -g.pad || j2 > g.nx + g.pad - 2) {
      j1 = j2 = 0;
      w = make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  *w_out = w;
  *o_out = ((j2 + g.pad) * g.L + j1 + g.pad) * g.nzp;
}

// one plane's pass table (weights hs | tails or folds ts | ranges 4 ints)
// into shared memory: half 0 = forward, 1 = adjoint
__device__ __forceinline__ void zs_table(const ZArgs& a, int set, int y, int half, float* Wt, int tid, int nth) {
  const int hs = a.g.hs, ts = a.g.ts;
  const float* Hrow = a.H + ((size_t)set * a.g.ny + y) * (2 * hs) + half * hs;
  const float* Erow = a.E + ((size_t)set * a.g.ny + y) * (2 * ts) + half * ts;
  for (int k = tid; k < hs + ts; k += nth) Wt[k] = k < hs ? Hrow[k] : Erow[k - hs];
  if (tid < 4) reinterpret_cast<int*>(Wt + hs + ts)[tid] = a.R[((size_t)set * a.g.ny + y) * 8 + 4 * half + tid];
}

// ------------------------------------------------------------------------
// k_zs_fz<NTH, W>: forward gather and z pass.  Shared memory (floats):
// [table hs + ts + 4][geoW tx float4][geoO tx int][ZB tx * ast][OB nz * tx]
template <int NTH, int W>
__global__ void __launch_bounds__(NTH) k_zs_fz(ZArgs a) {
  extern __shared__ float4 smem4[];
  const ZGeom& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nzp = g.nzp, hs = g.hs, ts = g.ts, tx = a.tx;
  float* const Wt = reinterpret_cast<float*>(smem4);
  float4* const geoW = reinterpret_cast<float4*>(Wt + hs + ts + 4);
  int* const geoO = reinterpret_cast<int*>(geoW + tx);
  float* const ZB = reinterpret_cast<float*>(geoO + tx);
  float* const OB = ZB + (size_t)tx * g.ast;
  const int tid = threadIdx.x, ast = g.ast, R0 = g.R0, hz = g.hz;
  const int ntx = nx / tx, nitems = a.nv * ny * ntx;
  const int nz4 = (nz + 3) / 4, units = tx * nz4, nzb = (nz + W - 1) / W, ztasks = tx * nzb, q4 = tx / 4;
  const size_t Lz = (size_t)g.L * nzp;
  const float rnz4 = 1.0f / nz4, rtx = 1.0f / tx, rq4 = 1.0f / q4;
  for (int k = tid; k < tx * ast; k += NTH) ZB[k] = 0.f;  // rows outside the data stay zero
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int xt = item % ntx, sy = item / ntx, slot = sy / ny, y = sy - slot * ny, X0 = xt * tx;
    const int v = a.vidx[slot], set = a.viewset[v];
    zs_table(a, set, y, 0, Wt, tid, NTH);
    if (tid < tx) zs_geometry(g, a.rot[v], X0 + tid, y, &geoW[tid], &geoO[tid]);
    __syncthreads();
    // rotated, attenuated columns into ZB (column x, rows R0 + z), two units a round
    const float* attp = a.att + (((size_t)v * ny + y) * nx + X0) * nzp;
    for (int u0 = tid; u0 < units; u0 += 2 * NTH) {
      float4 t[2][4], at[2];
      int xs[2], zs[2];
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const int u = min(u0 + j * NTH, units - 1);  // a repeated last unit stores the same values
        xs[j] = zdiv(u, rnz4);
        zs[j] = u - xs[j] * nz4;
        const float* p = a.img + geoO[xs[j]] + 4 * zs[j];
        t[j][0] = ld4(p);
        t[j][1] = ld4(p + nzp);
        t[j][2] = ld4(p + Lz);
        t[j][3] = ld4(p + Lz + nzp);
        at[j] = ld4(attp + (size_t)xs[j] * nzp + 4 * zs[j]);
      }
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        const float4 w = geoW[xs[j]];
        const float4 t0 = t[j][0], t1 = t[j][1], t2 = t[j][2], t3 = t[j][3];
        float4 o;
        o.x = __fmul_rn(fmaf(w.w, t3.x, fmaf(w.z, t2.x, fmaf(w.y, t1.x, __fmul_rn(w.x, t0.x)))), at[j].x);
        o.y = __fmul_rn(fmaf(w.w, t3.y, fmaf(w.z, t2.y, fmaf(w.y, t1.y, __fmul_rn(w.x, t0.y)))), at[j].y);
        o.z = __fmul_rn(fmaf(w.w, t3.z, fmaf(w.z, t2.z, fmaf(w.y, t1.z, __fmul_rn(w.x, t0.z)))), at[j].z);
        o.w = __fmul_rn(fmaf(w.w, t3.w, fmaf(w.z, t2.w, fmaf(w.y, t1.w, __fmul_rn(w.x, t0.w)))), at[j].w);
        st4(ZB + xs[j] * ast + R0 + 4 * zs[j], o);
      }
    }
    __syncthreads();
    // z pass: task (x, z block) -> OB rows z, column x
    const int2 rg = *reinterpret_cast<const int2*>(Wt + hs + ts);
    const float* ELz = Wt + hs;
    const float* ERz = ELz + hz;
    for (int t = tid; t < ztasks; t += NTH) {
      const int zb = zdiv(t, rtx), x = t - zb * tx, z0 = W * zb;
      float o[W];
#pragma unroll
      for (int k = 0; k < W; ++k) o[k] = 0.f;
      const float* col = ZB + x * ast;
      zpassw<W>(Wt, rg.x, rg.y, col + z0, o);
      if (z0 < hz) {
        const float e0 = col[R0];
#pragma unroll
        for (int k = 0; k < W; ++k)
          if (z0 + k < hz) o[k] = fmaf(ELz[z0 + k], e0, o[k]);
      }
      if (z0 + W > nz - hz) {
        const float e1 = col[R0 + nz - 1];
#pragma unroll
        for (int k = 0; k < W; ++k) {
          const int kk = nz - 1 - z0 - k;
          if (kk >= 0 && kk < hz) o[k] = fmaf(ERz[kk], e1, o[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < W; ++k)
        if (z0 + k < nz) OB[(z0 + k) * tx + x] = o[k];
    }
    __syncthreads();
    // the tile's rows -> Q[slot][y][z][X0 ..]
    float* Qp = a.Q + ((size_t)slot * ny + y) * nz * nx + X0;
    for (int e = tid; e < nz * q4; e += NTH) {
      const int z = zdiv(e, rq4), c = e - z * q4;
      st4(Qp + (size_t)z * nx + 4 * c, ld4(OB + z * tx + 4 * c));
    }
  }
}

// ------------------------------------------------------------------------
// k_zs_fx<NTH, W>: forward x pass and depth sum, one task of W outputs per
// thread and plane (tz * nx / W <= NTH; the host picks tz).  Shared memory
// (floats): 2 x [XB tz * bs (data columns C0..)][table hs + ts + 4].
template <int NTH, int W>
__global__ void __launch_bounds__(NTH, 1) k_zs_fx(ZArgs a) {
  extern __shared__ float4 smem4[];
  const ZGeom& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz, hs = g.hs, ts = g.ts, tz = a.tz, bs = g.bs, C0 = g.C0, hx = g.hx;
  const int bufsz = tz * bs + hs + ts + 4;
  float* const base = reinterpret_cast<float*>(smem4);
  const int tid = threadIdx.x;
  const int ntz = (nz + tz - 1) / tz, nitems = a.nv * a.nchunks * ntz, n4 = nx / 4, xbs = nx / W;
  const float rn4 = 1.0f / n4, rtz = 1.0f / tz;
  for (int k = tid; k < 2 * bufsz; k += NTH) base[k] = 0.f;  // padding columns stay zero
  __syncthreads();
  // this thread's task: row zl, x block xb
  const int xb = zdiv(tid, rtz), zl = tid - xb * tz, x0 = W * xb;
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int zt = item % ntz, sc = item / ntz, slot = sc / a.nchunks, ch = sc - slot * a.nchunks;
    const int Z0 = zt * tz, rows = min(tz, nz - Z0);
    const int y0 = ch * a.chunkY, y1 = min(ny, y0 + a.chunkY);
    const int v = a.vidx[slot], set = a.viewset[v];
    const bool mine = tid < tz * xbs && zl < rows;
    const int tot4 = rows * n4;
    auto src = [&](int y) { return a.Q + (((size_t)slot * ny + y) * nz + Z0) * nx; };
    // plane y0 straight into buffer 0
    {
      const float* Qp = src(y0);
      for (int e = tid; e < tot4; e += NTH) {
        const int z = zdiv(e, rn4), c = e - z * n4;
        st4(base + z * bs + C0 + 4 * c, ld4(Qp + (size_t)z * nx + 4 * c));
      }
      zs_table(a, set, y0, 0, base + tz * bs, tid, NTH);
    }
    __syncthreads();
    float acc[W];
#pragma unroll
    for (int k = 0; k < W; ++k) acc[k] = 0.f;
    for (int y = y0; y < y1; ++y) {
      float* const XB = base + ((y - y0) & 1) * bufsz;
      float* const XN = base + (((y - y0) & 1) ^ 1) * bufsz;
      const float* Wt = XB + tz * bs;
      // the next plane's rows into registers first (four float4 a thread at most)
      float4 pf[4];
      const bool more = y + 1 < y1;
      if (more) {
        const float* Qp = src(y + 1);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int e = tid + j * NTH;
          if (e < tot4) {
            const int z = zdiv(e, rn4), c = e - z * n4;
            pf[j] = ld4(Qp + (size_t)z * nx + 4 * c);
          }
        }
      }
      if (mine) {
        const int2 rg = *reinterpret_cast<const int2*>(Wt + hs + ts + 2);
        const float* ELx = Wt + hs + 2 * g.hz;
        const float* ERx = ELx + hx;
        const float* row = XB + zl * bs;
        zpassw<W>(Wt + g.zpw, rg.x, rg.y, row + x0, acc);
        if (x0 < hx) {
          const float e0 = row[C0];
#pragma unroll
          for (int k = 0; k < W; ++k)
            if (x0 + k < hx) acc[k] = fmaf(ELx[x0 + k], e0, acc[k]);
        }
        if (x0 + W > nx - hx) {
          const float e1 = row[C0 + nx - 1];
#pragma unroll
          for (int k = 0; k < W; ++k) {
            const int kk = nx - 1 - x0 - k;
            if (kk < hx) acc[k] = fmaf(ERx[kk], e1, acc[k]);
          }
        }
      }
      if (more) {
#pragma unroll
        for (int j = 0; j < 4; ++j) {
          const int e = tid + j * NTH;
          if (e < tot4) {
            const int z = zdiv(e, rn4), c = e - z * n4;
            st4(XN + z * bs + C0 + 4 * c, pf[j]);
          }
        }
        zs_table(a, set, y + 1, 0, XN + tz * bs, tid, NTH);
      }
      __syncthreads();
    }
    if (mine) {  // partial view of this chunk: part[slot][ch][z][x]
      float* o = a.part + (((size_t)slot * a.nchunks + ch) * nz + Z0 + zl) * nx + x0;
#pragma unroll
      for (int k = 0; k < W; k += 4) st4(o + k, make_float4(acc[k], acc[k + 1], acc[k + 2], acc[k + 3]));
    }
  }
}

// ------------------------------------------------------------------------
// k_zs_adj<NTH, W>: adjoint convolution of a tile of tx columns; item =
// (slot, column tile, depth chunk).  The view's columns X0 - C0 .. X0 + tx +
// xpw - C0 (zero outside the image) are loaded once per item as the tile's
// zero-padded lines, the same values at the same shifted positions as
// k_zadj's full rows; per plane the x pass (tx / W tasks a row) -> WB, the z
// pass times the attenuation -> T.  Shared memory (floats): [VB nz * tbs]
// [WB tx * ast: column x, data rows R0..][table hs + ts + 4], tbs =
// zstride4(tx + xpw).
template <int NTH, int W>
__global__ void __launch_bounds__(NTH) k_zs_adj(ZArgs a) {
  extern __shared__ float4 smem4[];
  const ZGeom& g = a.g;
  const int nx = g.nx, ny = g.ny, nz = g.nz, nzp = g.nzp, hs = g.hs, ts = g.ts, tx = a.tx;
  const int ast = g.ast, R0 = g.R0, C0 = g.C0, hz = g.hz, hx = g.hx, tbs = zstride4(tx + g.xpw);
  float* const VB = reinterpret_cast<float*>(smem4);
  float* const WB = VB + (size_t)nz * tbs;
  float* const Wt = WB + (size_t)tx * ast;
  const int tid = threadIdx.x;
  const int ntx = nx / tx, nitems = a.nv * ntx * a.nchunks, nzb = (nz + W - 1) / W;
  const int xbs = tx / W, xtasks = nz * xbs, ztasks = tx * nzb;
  const float rnz = 1.0f / nz, rtx = 1.0f / tx, rtbs = 1.0f / tbs;
  for (int k = tid; k < tx * ast; k += NTH) WB[k] = 0.f;  // rows outside the data stay zero
  for (int item = blockIdx.x; item < nitems; item += gridDim.x) {
    const int ch = item % a.nchunks, st = item / a.nchunks, slot = st / ntx, xt = st - slot * ntx;
    const int X0 = xt * tx, y0 = ch * a.chunkY, y1 = min(ny, y0 + a.chunkY);
    const int v = a.vidx[slot], set = a.viewset[v];
    // the tile's lines: VB[z][c] = view[z][X0 + c - C0] inside the image, else
    // zero (the previous item's last pass ended at a barrier)
    const float* V = a.views + (size_t)slot * nz * nx;
    for (int e = tid; e < nz * tbs; e += NTH) {
      const int z = zdiv(e, rtbs), c = e - z * tbs, xg = X0 + c - C0;
      VB[e] = (xg >= 0 && xg < nx) ? V[(size_t)z * nx + xg] : 0.f;
    }
    for (int y = y0; y < y1; ++y) {
      zs_table(a, set, y, 1, Wt, tid, NTH);
      __syncthreads();
      // x pass: task (z, x block) -> WB column x, row R0 + z
      {
        const int2 rg = *reinterpret_cast<const int2*>(Wt + hs + ts + 2);
        const float* cLx = Wt + hs;
        const float* cRx = cLx + hx;
        for (int t = tid; t < xtasks; t += NTH) {
          const int xb = zdiv(t, rnz), z = t - xb * nz, x0 = W * xb;
          const float* row = VB + z * tbs;
          float o[W];
#pragma unroll
          for (int k = 0; k < W; ++k) o[k] = 0.f;
          zpassw<W>(Wt + g.zpw, rg.x, rg.y, row + x0, o);
          if (X0 + x0 == 0) o[0] += zfold(cLx, row + C0, 1, hx);
          if (X0 + x0 + W == nx) o[W - 1] += zfold(cRx, row + C0 + x0 + W - 1, -1, hx);
          float* w = WB + x0 * ast + R0 + z;
#pragma unroll
          for (int k = 0; k < W; ++k) w[k * ast] = o[k];
        }
      }
      __syncthreads();
      // z pass: task (x, z block) -> T column (X0 + x, y) of the slot
      {
        const int2 rg = *reinterpret_cast<const int2*>(Wt + hs + ts);
        const float* cLz = Wt + hs + 2 * hx;
        const float* cRz = cLz + hz;
        const float* attv = a.att + (((size_t)v * ny + y) * nx + X0) * nzp;
        float* Tp = a.T + (((size_t)slot * ny + y) * nx + X0) * nzp;
        for (int t = tid; t < ztasks; t += NTH) {
          const int zb = zdiv(t, rtx), x = t - zb * tx, z0 = W * zb;
          float4 at[W / 4];
#pragma unroll
          for (int k = 0; k < W / 4; ++k) at[k] = ld4(attv + (size_t)x * nzp + z0 + 4 * k);
          const float* col = WB + x * ast;
          float o[W];
#pragma unroll
          for (int k = 0; k < W; ++k) o[k] = 0.f;
          zpassw<W>(Wt, rg.x, rg.y, col + z0, o);
          if (z0 == 0) o[0] += zfold(cLz, col + R0, 1, hz);
          if (z0 <= nz - 1 && nz - 1 < z0 + W) {
            const int kz = nz - 1 - z0;
            const float s = zfold(cRz, col + R0 + nz - 1, -1, hz);
#pragma unroll
            for (int k = 0; k < W; ++k)
              if (k == kz) o[k] += s;
          }
          float* dst = Tp + (size_t)x * nzp + z0;
#pragma unroll
          for (int k = 0; k < W / 4; ++k)
            st4(dst + 4 * k, make_float4(__fmul_rn(at[k].x, o[4 * k]), __fmul_rn(at[k].y, o[4 * k + 1]),
                                         __fmul_rn(at[k].z, o[4 * k + 2]), __fmul_rn(at[k].w, o[4 * k + 3])));
        }
      }
      __syncthreads();
    }
  }
}

}  // namespace spect
