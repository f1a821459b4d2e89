// HEVI small-step kernels: 3-D/2-D divergence damping, pressure gradient,
// vp0 source terms + tridiagonal matrix, the acoustic-loop path1 update and
// vi_main (flux convergences + Thomas solve + energy update).
#pragma once
#include "nc_large.cuh"

namespace nc {

// ---------------------------------------------------------------------------
// 3-D divergence damping operator (kernels/oprt3ddivdamp.py:85-173)
// ---------------------------------------------------------------------------
template <class R>
struct Four { const R* f[4]; };   // rhogvx, rhogvy, rhogvz, rhogw
template <class R>
struct Three { R* f[3]; };
template <class R>
struct CThree { const R* f[3]; };

// the six-edge divergence-damping combination for direction d at (i,j)
// (kernels/oprtdivdamp.py:110-120)
template <class R>
__device__ __forceinline__ R ddivd(int i, int j, int l, int d, const R aTI, const R aTJ,
                                        const R bTI, const R cTJ, const R cTI, const R dTJ) {
  return P2(CG.coef_diff, d * 6 + 0, i, j, l) * (aTI + aTJ) + P2(CG.coef_diff, d * 6 + 1, i, j, l) * (aTJ + bTI) +
         P2(CG.coef_diff, d * 6 + 2, i, j, l) * (bTI + cTJ) + P2(CG.coef_diff, d * 6 + 3, i, j, l) * (cTJ + cTI) +
         P2(CG.coef_diff, d * 6 + 4, i, j, l) * (cTI + dTJ) + P2(CG.coef_diff, d * 6 + 5, i, j, l) * (dTJ + aTI);
}

// Tiled 3-D divergence damping: one block per DD_DX x DD_DY tile of output
// cells of one region, marching upward in k.  Per level the block stages the
// haloed tile of RGAM-scaled momentum and the vertical mass flux rwv(k+1) in
// shared memory (rwv(k) is kept from the level below), evaluates every
// triangle value once, applies the singular-point fix, then each thread forms
// its cell's three components.  Per triangle: the RGAM-weighted momenta at
// its three vertices against coef_intp plus the vertical flux difference
// ((rwv(k+1) summed over the vertices) - (rwv(k) summed)) / 3 * rdgz(k)
// (kernels/oprt3ddivdamp.py:50-173); the rwv sums and coefficient products
// are added left to right in the reference's order.
#ifndef DD_DX
#define DD_DX 32
#endif
#ifndef DD_DY
#define DD_DY 8
#endif
// resident blocks per SM for a register budget of n blocks of 256 threads
#define DD_MINB(n) ((n) * 256 / (DD_DX * DD_DY) > 0 ? (n) * 256 / (DD_DX * DD_DY) : 1)
// The tile's k-invariant coefficients are read once per block instead of
// once per level: the triangle weights coef_intp (18 planes) staged in shared
// memory, the cell's coef_diff (18) held in registers (CDR) or read per
// level.  Dynamic shared memory dd3d_m_smem<R>().
template <class R>
constexpr int dd3d_m_smem() {
  return (18 * (DD_DX + 1) * (DD_DY + 1) + 5 * (DD_DX + 2) * (DD_DY + 2) + 2 * (DD_DX + 1) * (DD_DY + 1)) *
         (int)sizeof(R);
}
#ifndef DD_M_MINB
#define DD_M_MINB 2
#endif
// The next level's staging writes s_vm and the rwv buffer of the level below,
// which only this level's triangle pass reads (done before its second
// barrier), and the next level's triangle pass writes s_ti / s_tj only after
// the next first barrier, which every thread reaches after its cell pass: no
// barrier is needed at the end of a level, and the corner tile alone waits
// for its singular-point fix.

template <class R, bool CDR>
__global__ void __launch_bounds__(DD_DX * DD_DY, DD_MINB(NC_MINB(R, DD_M_MINB, 4))) k_dd3d_m(Four<R> v, Three<R> out) {
  constexpr int PX = DD_DX + 2, PY = DD_DY + 2, NP = PX * PY;
  constexpr int TX = DD_DX + 1, TY = DD_DY + 1, NT = TX * TY;
  extern __shared__ __align__(16) unsigned char dd_smem[];
  R* s_ci = reinterpret_cast<R*>(dd_smem);   // [18][NT] coef_intp of each triangle
  R* s_vm = s_ci + 18 * NT;                    // [3][NP]
  R* s_rw = s_vm + 3 * NP;                     // [2][NP]
  R* s_ti = s_rw + 2 * NP;                     // [NT]
  R* s_tj = s_ti + NT;                         // [NT]
  const int l = blockIdx.z;
  const int i0 = 1 + blockIdx.x * DD_DX, j0 = 1 + blockIdx.y * DD_DY;
  const int G = cD.G, gmax = cD.G - 2;
  const int tid = threadIdx.x, tx = tid % DD_DX, ty = tid / DD_DX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= gmax) && (j <= gmax);
  const int n = cD.npti;
  const R* cz = CG.C2WGz;
  for (int p = tid; p < NT; p += blockDim.x) {
    const int ii = i0 - 1 + p % TX, jj = j0 - 1 + p / TX;
    const bool ok = ii <= G - 2 && jj <= G - 2;
#pragma unroll
    for (int m = 0; m < 18; ++m) s_ci[m * NT + p] = ok ? P2c(CG.coef_intp, m, ii, jj, l) : R(0.0);
  }
  R cd[CDR ? 18 : 1];
  if (CDR && own) {
#pragma unroll
    for (int m = 0; m < (CDR ? 18 : 1); ++m) cd[m] = P2c(CG.coef_diff, m, i, j, l);
  }
  for (int p = tid; p < NP; p += blockDim.x) s_rw[p] = R(0.0);   // rwv(kmin) = 0
  int cur = 0;
  for (int k = cD.kmin; k <= cD.kmax; ++k) {
    const bool up = (k + 1 <= cD.kmax);   // rwv(k+1) = 0 above kmax
    for (int p = tid; p < NP; p += blockDim.x) {
      const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
      R a = R(0.0), b = R(0.0), c = R(0.0), r = R(0.0);
      if (ii < G && jj < G) {
        const int q = ix(ii, jj, k, l);
        const R f0 = v.f[0][q], f1 = v.f[1][q], f2 = v.f[2][q];
        const R rg = gam_at(CG.RGAM, q);
        a = f0 * rg;
        b = f1 * rg;
        c = f2 * rg;
        if (up) {
          const int qp = q + cD.planei;   // level k+1
          const R h = cz[qp] * v.f[0][qp] + cz[n + qp] * f0 + cz[2 * n + qp] * v.f[1][qp] +
                      cz[3 * n + qp] * f1 + cz[4 * n + qp] * v.f[2][qp] + cz[5 * n + qp] * f2;
          r = h * gam_at(CG.RGAMH, qp) + v.f[3][qp] * CG.RGSQRTH[qp];
        }
      }
      s_vm[p] = a;
      s_vm[NP + p] = b;
      s_vm[2 * NP + p] = c;
      s_rw[(cur ^ 1) * NP + p] = r;
    }
    __syncthreads();
    const R rdz = CC.rdgz[k];
    const R* rU = s_rw + (cur ^ 1) * NP;
    const R* rD = s_rw + cur * NP;
    for (int p = tid; p < NT; p += blockDim.x) {
      const int px = p % TX, py = p / TX;
      const int a = py * PX + px, b = a + 1, c = a + PX + 1, d = a + PX;
      auto C = [&](int dir, int pt, int t) { return s_ci[((dir * 3 + pt) * 2 + t) * NT + p]; };
      const R wTI = div3((rU[a] + rU[b] + rU[c]) - (rD[a] + rD[b] + rD[c])) * rdz;
      const R wTJ = div3((rU[a] + rU[c] + rU[d]) - (rD[a] + rD[c] + rD[d])) * rdz;
      const R* v0 = s_vm;
      const R* v1 = s_vm + NP;
      const R* v2 = s_vm + 2 * NP;
      R sTI = C(0, 0, 0) * v0[a] + C(0, 1, 0) * v0[b] + C(0, 2, 0) * v0[c] + C(1, 0, 0) * v1[a] +
              C(1, 1, 0) * v1[b] + C(1, 2, 0) * v1[c] + C(2, 0, 0) * v2[a] + C(2, 1, 0) * v2[b] +
              C(2, 2, 0) * v2[c] + wTI;
      R sTJ = C(0, 0, 1) * v0[a] + C(0, 1, 1) * v0[c] + C(0, 2, 1) * v0[d] + C(1, 0, 1) * v1[a] +
              C(1, 1, 1) * v1[c] + C(1, 2, 1) * v1[d] + C(2, 0, 1) * v2[a] + C(2, 1, 1) * v2[c] +
              C(2, 2, 1) * v2[d] + wTJ;
      const int ii = i0 - 1 + px, jj = j0 - 1 + py;
      if (!(ii <= G - 2 && jj <= G - 2)) sTI = sTJ = R(0.0);
      s_ti[p] = sTI;
      s_tj[p] = sTJ;
    }
    __syncthreads();
    if (i0 == 1 && j0 == 1) {   // singular-point fix at the (0,0) triangle (block-uniform branch)
      if (tid == 0) s_ti[0] = s_ti[0] * (R)CG.pntmask[l * 2 + 0] + s_tj[1] * (R)CG.pntmask[l * 2 + 1];
      __syncthreads();
    }
    if (own) {
      const int ta = (ty + 1) * TX + (tx + 1);   // triangle (i, j)
      const R aTI = s_ti[ta], aTJ = s_tj[ta];
      const R bTI = s_ti[ta - 1];            // (i-1, j)
      const R cTI = s_ti[ta - TX - 1], cTJ = s_tj[ta - TX - 1];   // (i-1, j-1)
      const R dTJ = s_tj[ta - TX];           // (i, j-1)
      const int q = ix(i, j, k, l);
      auto D = [&](int m) { return CDR ? cd[CDR ? m : 0] : P2c(CG.coef_diff, m, i, j, l); };
#pragma unroll
      for (int d = 0; d < 3; ++d)
        out.f[d][q] = D(d * 6 + 0) * (aTI + aTJ) + D(d * 6 + 1) * (aTJ + bTI) + D(d * 6 + 2) * (bTI + cTJ) +
                      D(d * 6 + 3) * (cTJ + cTI) + D(d * 6 + 4) * (cTI + dTJ) + D(d * 6 + 5) * (dTJ + aTI);
    }
    cur ^= 1;
  }
}

// Block -> (level, tile, region) of the per-level tiled kernels: the level
// is the fastest block index so that blocks sharing a tile's haloed data at
// neighbouring levels run together and meet in L2.
struct TileLv {
  int k, l, i0, j0;
};
template <int TDX, int TDY>
__device__ __forceinline__ TileLv tile_level(int kbase) {
  const int ntx = (cD.G - 2 + TDX - 1) / TDX;
  TileLv t;
  t.k = kbase + (int)blockIdx.x;
  t.l = (int)blockIdx.z;
  t.i0 = 1 + ((int)blockIdx.y % ntx) * TDX;
  t.j0 = 1 + ((int)blockIdx.y / ntx) * TDY;
  return t;
}

// pole 3-D divergence damping (kernels/oprt3ddivdamp.py:176-237)
template <class R>
__global__ void k_dd3d_pl(Four<R> v, Three<R> out) {
  int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.KA * cD.LP) return;
  int k = t / cD.LP, lp = t % cD.LP;
  for (int g = 0; g < 6; ++g)
    for (int d = 0; d < 3; ++d) out.f[d][ipl(g, k, lp)] = R(0.0);
  if (k < cD.kmin || k > cD.kmax) return;
  auto rw = [&](int g, int kk) -> R {
    if (kk <= cD.kmin || kk > cD.kmax) return R(0.0);
    int q = ipl(g, kk, lp), qm = ipl(g, kk - 1, lp);
    const R* cz = CG.C2WGz_pl;
    R h = cz[q * 6 + 0] * v.f[0][q] + cz[q * 6 + 1] * v.f[0][qm] + cz[q * 6 + 2] * v.f[1][q] +
               cz[q * 6 + 3] * v.f[1][qm] + cz[q * 6 + 4] * v.f[2][q] + cz[q * 6 + 5] * v.f[2][qm];
    return h * gam_at(CG.RGAMH_pl, q) + v.f[3][q] * CG.RGSQRTH_pl[q];
  };
  R vm[6][3];
  for (int g = 0; g < 6; ++g) {
    int q = ipl(g, k, lp);
    for (int d = 0; d < 3; ++d) vm[g][d] = v.f[d][q] * gam_at(CG.RGAM_pl, q);
  }
  R sclt[5];
  for (int v_ = 1; v_ <= 5; ++v_) {
    int vp1 = (v_ == 5) ? 1 : v_ + 1;
    R sw = div3((rw(0, k + 1) + rw(v_, k + 1) + rw(vp1, k + 1)) - (rw(0, k) + rw(v_, k) + rw(vp1, k))) * CC.rdgz[k];
    const R* cI = CG.coef_intp_pl + (v_ * cD.LP + lp) * 9;
    sclt[v_ - 1] = cI[0] * vm[0][0] + cI[1] * vm[v_][0] + cI[2] * vm[vp1][0] + cI[3] * vm[0][1] + cI[4] * vm[v_][1] +
                   cI[5] * vm[vp1][1] + cI[6] * vm[0][2] + cI[7] * vm[v_][2] + cI[8] * vm[vp1][2] + sw;
  }
  for (int d = 0; d < 3; ++d) {
    R row = R(0.0);
    for (int v_ = 1; v_ <= 5; ++v_) {
      int vm1 = (v_ == 1) ? 5 : v_ - 1;
      R pair = sclt[vm1 - 1] + sclt[v_ - 1];
      R tv = CG.coef_diff_pl[(v_ * cD.LP + lp) * 3 + d] * pair;
      row = (v_ == 1) ? tv : row + tv;
    }
    out.f[d][ipl(0, k, lp)] = row;
  }
}

// ---------------------------------------------------------------------------
// post-COMM 2-D divergence damping (kernels/divdamppostcomm.py:29-81):
// gd = coef * OPRT_divdamp(-vtmp2), then horizontalize (interior).
// ---------------------------------------------------------------------------
template <class R>
__device__ void divdamp2d_at(const CThree<R>& vt, int i, int j, int k, int l, R gd[3]) {
  if (!interior(i, j)) {
    for (int d = 0; d < 3; ++d) gd[d] = CC.divdamp_coef * R(0.0);
    return;
  }
  auto sc = [&](int ii, int jj, R& sTI, R& sTJ) {
    int a = ix(ii, jj, k, l), b = ix(ii + 1, jj, k, l), c = ix(ii + 1, jj + 1, k, l), d = ix(ii, jj + 1, k, l);
    auto C = [&](int dir, int p, int t) { return P2(CG.coef_intp, (dir * 3 + p) * 2 + t, ii, jj, l); };
    R x0 = -vt.f[0][a], x1 = -vt.f[0][b], x2 = -vt.f[0][c], x3 = -vt.f[0][d];
    R y0 = -vt.f[1][a], y1 = -vt.f[1][b], y2 = -vt.f[1][c], y3 = -vt.f[1][d];
    R z0 = -vt.f[2][a], z1 = -vt.f[2][b], z2 = -vt.f[2][c], z3 = -vt.f[2][d];
    sTI = C(0, 0, 0) * x0 + C(0, 1, 0) * x1 + C(0, 2, 0) * x2 + C(1, 0, 0) * y0 + C(1, 1, 0) * y1 + C(1, 2, 0) * y2 +
          C(2, 0, 0) * z0 + C(2, 1, 0) * z1 + C(2, 2, 0) * z2;
    sTJ = C(0, 0, 1) * x0 + C(0, 1, 1) * x2 + C(0, 2, 1) * x3 + C(1, 0, 1) * y0 + C(1, 1, 1) * y2 + C(1, 2, 1) * y3 +
          C(2, 0, 1) * z0 + C(2, 1, 1) * z2 + C(2, 2, 1) * z3;
  };
  R aTI, aTJ, bTI, bTJ, cTI, cTJ, dTI, dTJ;
  sc(i, j, aTI, aTJ);
  sc(i - 1, j, bTI, bTJ);
  sc(i - 1, j - 1, cTI, cTJ);
  sc(i, j - 1, dTI, dTJ);
  R o[3];
  for (int d = 0; d < 3; ++d) o[d] = CC.divdamp_coef * ddivd(i, j, l, d, aTI, aTJ, bTI, cTJ, cTI, dTJ);
  horiz_reg(i, j, l, o[0], o[1], o[2]);
  gd[0] = o[0]; gd[1] = o[1]; gd[2] = o[2];
}

// pole 2-D divergence damping of -vtmp2 at (g,k,lp) (kernels/oprtdivdamp.py:125-173
// then horizontalize over all g)
template <class R>
__device__ void divdamp2d_pl_at(const CThree<R>& vt, int g, int k, int lp, R gd[3]) {
  R o[3] = {R(0.0), R(0.0), R(0.0)};
  if (g == 0) {
    R vv[6][3];
    for (int q = 0; q < 6; ++q)
      for (int d = 0; d < 3; ++d) vv[q][d] = -vt.f[d][ipl(q, k, lp)];
    R sclt[5];
    for (int v_ = 1; v_ <= 5; ++v_) {
      int vp1 = (v_ == 5) ? 1 : v_ + 1;
      const R* cI = CG.coef_intp_pl + (v_ * cD.LP + lp) * 9;
      sclt[v_ - 1] = cI[0] * vv[0][0] + cI[1] * vv[v_][0] + cI[2] * vv[vp1][0] + cI[3] * vv[0][1] +
                     cI[4] * vv[v_][1] + cI[5] * vv[vp1][1] + cI[6] * vv[0][2] + cI[7] * vv[v_][2] +
                     cI[8] * vv[vp1][2];
    }
    for (int d = 0; d < 3; ++d) {
      R row = R(0.0);
      for (int v_ = 1; v_ <= 5; ++v_) {
        int vm1 = (v_ == 1) ? 5 : v_ - 1;
        R tv = CG.coef_diff_pl[(v_ * cD.LP + lp) * 3 + d] * (sclt[vm1 - 1] + sclt[v_ - 1]);
        row = (v_ == 1) ? tv : row + tv;
      }
      o[d] = row;
    }
  }
  for (int d = 0; d < 3; ++d) o[d] = CC.divdamp_coef * o[d];
  horiz_pl(g, lp, o[0], o[1], o[2]);
  gd[0] = o[0]; gd[1] = o[1]; gd[2] = o[2];
}

// ---------------------------------------------------------------------------
// pressure gradient (kernels/presgrad.py:126-265): horizontal part at level
// k with the first-layer remedy and the tangent-plane projection.
// P(ii,jj,kk) gives the pressure; returns Pgrad (3 comps).
// ---------------------------------------------------------------------------
template <class R, class PF>
__device__ void presgrad_reg(int i, int j, int k, int l, const Col& c, const MetT<R>& m, PF P, R out[3]) {
  const int kmin = cD.kmin, kmax = cD.kmax;
  out[0] = out[1] = out[2] = R(0.0);
  if (k >= kmin && k <= kmax) {
    const int kk = (k == kmin) ? kmin + 1 : k;
    R gh[3] = {R(0.0), R(0.0), R(0.0)};
    if (interior(i, j)) grad7(i, j, kk, l, [&](int ii, int jj, int k2) { return P(ii, jj, k2) * gam_at(CG.RGAM, ix(ii, jj, k2, l)); }, gh);
    auto pvmh = [&](int k2, int d) {
      return (mc(m.C2WGz, c, 2 * d, 6, k2) * P(i, j, k2) + mc(m.C2WGz, c, 2 * d + 1, 6, k2) * P(i, j, k2 - 1)) *
             gam_at(m.RGAMH, c.at(k2));
    };
    for (int d = 0; d < 3; ++d) out[d] = gh[d] + (pvmh(kk + 1, d) - pvmh(kk, d)) * CC.rdgz[kk];
  }
  if (interior(i, j)) horiz_reg(i, j, l, out[0], out[1], out[2]);
}

template <class R, class PF>
__device__ void presgrad_pl(int g, int k, int lp, const Col& c, const MetT<R>& m, PF P, R out[3]) {
  const int kmin = cD.kmin, kmax = cD.kmax;
  out[0] = out[1] = out[2] = R(0.0);
  if (k >= kmin && k <= kmax) {
    const int kk = (k == kmin) ? kmin + 1 : k;
    R gh[3] = {R(0.0), R(0.0), R(0.0)};
    if (g == 0) {
      for (int d = 0; d < 3; ++d) {
        R row = R(0.0);
        for (int v_ = 0; v_ < 6; ++v_) {
          R pvm = P(v_, kk) * gam_at(CG.RGAM_pl, ipl(v_, kk, lp)) * R(1.0);
          R tv = CG.coef_grad_pl[(v_ * cD.LP + lp) * 3 + d] * pvm;
          row = (v_ == 0) ? tv : row + tv;
        }
        gh[d] = row;
      }
    }
    auto pvmh = [&](int k2, int d) {
      return (mc(m.C2WGz, c, 2 * d, 6, k2) * P(g, k2) + mc(m.C2WGz, c, 2 * d + 1, 6, k2) * P(g, k2 - 1)) *
             gam_at(m.RGAMH, c.at(k2));
    };
    for (int d = 0; d < 3; ++d) out[d] = gh[d] + (pvmh(kk + 1, d) - pvmh(kk, d)) * CC.rdgz[kk];
  }
  horiz_pl(g, lp, out[0], out[1], out[2]);
}

// vertical pressure gradient (kernels/presgrad.py:196-204)
template <class R, class PF>
__device__ __forceinline__ R presgradw(const Col& c, const MetT<R>& m, int k, PF Pk) {
  if (k < cD.kmin + 1 || k > cD.kmax) return R(0.0);
  int p = c.at(k), pm = c.at(k - 1);
  return gam_at(m.GAM2H, p) * (Pk(k) * m.RGSGAM2[p] - Pk(k - 1) * m.RGSGAM2[pm]) * CC.rdgzh[k];
}

// flux convergence at level k of a regional or pole column given the
// horizontal divergence value (zero on the halo) and the flux accessors
// (kernels/fluxconv.py:111-208, vflag 1 or 0)
template <class R, class FH, class FW>
__device__ __forceinline__ R fluxconv_col(const Col& c, const MetT<R>& m, int k, typename Id<R>::type div,
                                          typename Id<R>::type vflag, FH fh, FW fw) {
  if (k < cD.kmin || k > cD.kmax) return R(0.0);
  auto vmh = [&](int kk) -> R {
    if (kk <= cD.kmin || kk > cD.kmax) return R(0.0);
    R h = vmh_horiz(c, m, kk, fh);
    return h + vflag * fw(kk) * m.RGSQRTH[c.at(kk)];
  };
  return -div - (vmh(k + 1) - vmh(k)) * CC.rdgz[k];
}

// pole divergence row of (fx,fy,fz)*RGAM at level k (kernels/fluxconv.py:81-108)
template <class R, class F>
__device__ __forceinline__ R div_pl(int lp, int k, F f) {
  R row = R(0.0);
  for (int v_ = 0; v_ < 6; ++v_) {
    int q = ipl(v_, k, lp);
    R rg = gam_at(CG.RGAM_pl, q);
    R vx = f(q, 0) * rg, vy = f(q, 1) * rg, vz = f(q, 2) * rg;
    const R* cd = CG.coef_div_pl + (v_ * cD.LP + lp) * 3;
    R pv = cd[0] * vx + cd[1] * vy + cd[2] * vz;
    row = (v_ == 0) ? pv : row + pv;
  }
  return row;
}

// ---------------------------------------------------------------------------
// vp0: small-step source terms, g_TEND of the small step, the vertical
// implicit matrix and ethtot0 (mod_vi.py:295-878 numpy path,
// kernels/vimatrix.py:67-136, kernels/vimain.py:195-239)
// ---------------------------------------------------------------------------
template <class R>
struct Vp0Args {
  Prog<R> P;                    // PROG (post BNDCND)
  const R *vx, *vy, *vz, *eth;
  const double *pregd, *rhogd;  // float64 in both forms
  CThree<R> vt;                 // post-COMM 3-D divdamp of PROG
  const R* gT0[6];              // large-step tendency
  R* gT[6];                     // out: small-step tendency
  double *Mc, *Mu, *Ml;         // float64 in both forms
  R* ethtot0;
  double dt;                    // small-step dt
};

// One pole column of vp0.  In the mixed form the horizontal operators run in
// float32 (R) and the vertical part -- buoyancy and vertical pressure gradient
// of the float64 deviations, gz, the implicit matrix and the vertical-momentum
// tendency -- in float64, as in the regional column kernel k_vp0_cr.
template <class R, bool POLE>
__device__ void vp0_column(const Vp0Args<R>& a, int i, int j, int l, int g, int lp) {
  const Col c = POLE ? col_pl(g, lp) : col_reg(i, j, l);
  const MetT<R> m = met_of<R>(POLE);
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  const R* const* P = a.P.v;
  const double dt = a.dt;
  // column-local half-level values (float64)
  auto rhog_h = [&](int k) -> double {
    int kk = (k < kmin) ? kmin : k;
    return (double)mc(m.C2W, c, 0, 2, kk) * (double)P[0][c.at(kk)] +
           (double)mc(m.C2W, c, 1, 2, kk) * (double)P[0][c.at(kk - 1)];
  };
  auto eth_h = [&](int k) -> double {
    int kk = (k < kmin) ? kmin : k;
    return cC.afact[kk] * (double)a.eth[c.at(kk)] + cC.bfact[kk] * (double)a.eth[c.at(kk - 1)];
  };
  auto dbuo = [&](int k) -> double {
    if (k < kmin + 1 || k > kmax) return 0.0;
    return -cC.GRAV * ((double)mc(m.C2W, c, 0, 2, k) * a.rhogd[c.at(k)] +
                       (double)mc(m.C2W, c, 1, 2, k) * a.rhogd[c.at(k - 1)]);
  };
  auto dpgw = [&](int k) -> double {
    if (k < kmin + 1 || k > kmax) return 0.0;
    const int p = c.at(k), pm = c.at(k - 1);
    return (double)gam_at(m.GAM2H, p) *
           (a.pregd[p] * (double)m.RGSGAM2[p] - a.pregd[pm] * (double)m.RGSGAM2[pm]) * cC.rdgzh[k];
  };
  auto gz = [&](int k) -> double { return cC.GRAV - (dpgw(k) - dbuo(k)) / rhog_h(k); };
  auto pwh = [&](int k) -> R { return R(-gz(k) * (double)P[4][c.at(k)]); };
  auto PF = [&](int k, int d) -> R { return P[1 + d][c.at(k)]; };
  auto PEF = [&](int k, int d) -> R { return P[1 + d][c.at(k)] * a.eth[c.at(k)]; };
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    // horizontal divergences
    R div1 = R(0.0), div2 = R(0.0);
    if (!POLE) {
      if (interior(i, j)) {
        div1 = div7<R>(i, j, k, l, [&](int ii, int jj, int kk, int d) {
          int q = ix(ii, jj, kk, l);
          return P[1 + d][q] * gam_at(CG.RGAM, q);
        });
        div2 = div7<R>(i, j, k, l, [&](int ii, int jj, int kk, int d) {
          int q = ix(ii, jj, kk, l);
          return (P[1 + d][q] * a.eth[q]) * gam_at(CG.RGAM, q);
        });
      }
    } else if (g == 0) {
      div1 = div_pl<R>(lp, k, [&](int q, int d) { return P[1 + d][q]; });
      div2 = div_pl<R>(lp, k, [&](int q, int d) { return P[1 + d][q] * a.eth[q]; });
    }
    R drhog = fluxconv_col(c, m, k, div1, R(1.0), PF, [&](int kk) { return P[4][c.at(kk)]; });
    R drhoge = fluxconv_col(c, m, k, div2, R(1.0), PEF, [&](int kk) {
      int q = c.at(kk);
      return P[4][q] * (CC.afact[kk] * a.eth[q] + CC.bfact[kk] * a.eth[c.at(kk - 1)]);
    });
    R dd[3], dpg[3];
    if (!POLE) {
      divdamp2d_at(a.vt, i, j, k, l, dd);
      presgrad_reg(i, j, k, l, c, m, [&](int ii, int jj, int kk) { return R(a.pregd[ix(ii, jj, kk, l)]); }, dpg);
    } else {
      divdamp2d_pl_at(a.vt, g, k, lp, dd);
      presgrad_pl(g, k, lp, c, m, [&](int gg, int kk) { return R(a.pregd[ipl(gg, kk, lp)]); }, dpg);
    }
    R pw = R(0.0);
    if (k >= kmin && k <= kmax)
      pw = a.vx[p] * dpg[0] + a.vy[p] * dpg[1] + a.vz[p] * dpg[2] + mc(m.W2C, c, 0, 2, k) * pwh(k + 1) +
           mc(m.W2C, c, 1, 2, k) * pwh(k);
    a.gT[0][p] = a.gT0[0][p] + drhog;
    a.gT[1][p] = a.gT0[1][p] - dpg[0] + dd[0] + R(0.0);
    a.gT[2][p] = a.gT0[2][p] - dpg[1] + dd[1] + R(0.0);
    a.gT[3][p] = a.gT0[3][p] - dpg[2] + dd[2] + R(0.0);
    a.gT[4][p] = R((double)a.gT0[4][p] + 0.0 * cC.alpha - dpgw(k) + dbuo(k));
    a.gT[5][p] = a.gT0[5][p] + drhoge + pw;
    // vertical implicit matrix on k = kmin+1..kmax (float64)
    if (k >= kmin + 1 && k <= kmax) {
      const double GCVovR = cC.GRAV * cC.CVdry / cC.Rdry;
      const double ACVovRt2 = cC.alpha * cC.CVdry / cC.Rdry / (dt * dt);
      int pm = c.at(k - 1), pp = c.at(k + 1);
      double rg = cC.rdgz[k], rgm = cC.rdgz[k - 1];
      double Ca = ((double)m.RGSGAM2[p] * rg + (double)m.RGSGAM2[pm] * rgm) * (double)gam_at(m.GAM2H, p);
      double Cb = cC.dfact[k] - cC.cfact[k - 1];
      double Cu1 = (double)m.RGSGAM2[p] * rg * (double)gam_at(m.GAM2H, pp);
      double rgh2 = (double)gam_at(m.RGAMH, p) * (double)gam_at(m.RGAMH, p);
      double Cu2 = (double)gam_at(m.GAM2H, pp) * rgh2 * GCVovR;
      double Cl1 = (double)m.RGSGAM2[p] * rg * (double)gam_at(m.GAM2H, pm);
      double Cl2 = (double)gam_at(m.GAM2H, pm) * rgh2 * GCVovR;
      double rgh = cC.rdgzh[k];
      a.Mc[p] = ACVovRt2 / (double)m.RGSQRTH[p] + rgh * (Ca * eth_h(k) - Cb * (gz(k) + GCVovR));
      a.Mu[p] = -rgh * (Cu1 * eth_h(k + 1) + cC.cfact[k] * (gz(k + 1) + Cu2));
      a.Ml[p] = -rgh * (Cl1 * eth_h(k - 1) - cC.dfact[k - 1] * (gz(k - 1) + Cl2));
    }
    // total energy at the start of the small steps
    R kin0 = rhogkin_at(c, m, k, [&](int kk, int comp) { return P[comp][c.at(kk)]; });
    a.ethtot0[p] = a.eth[p] + kin0 / P[0][p] + m.PHI[p];
  }
}

// Horizontal terms of vp0, tiled like k_path1_l: for interior cells and
// levels kmin..kmax, the divergences of RGAM*rhogv and RGAM*rhogv*eth
// (div1, div2), the 2-D divergence damping of -vtmp2 (dd) and the pressure
// gradient of pregd (dpg), written to eight work fields for the column kernel.
template <class R>
struct Vp0H {
  R* out[8];               // div1, div2, dd x/y/z, dpg x/y/z
};

// vp0 horizontal terms, one block per (level, tile).
// vp0 keeps a 32x8 tile: its staged fields need more than the 48 KB of
// static shared memory at larger tiles
#define VP_DX 32
#define VP_DY 8
template <class R>
__global__ void __launch_bounds__(VP_DX * VP_DY, NC_MINB(R, 4, NC_F32_VP0H)) k_vp0_hl(Vp0Args<R> a, Vp0H<R> h) {
  constexpr int PX = VP_DX + 2, PY = VP_DY + 2, TX = VP_DX + 1, TY = VP_DY + 1;
  __shared__ R s_m[3][PY * PX];    // RGAM * rhogv
  __shared__ R s_e[3][PY * PX];    // RGAM * rhogv * eth
  __shared__ R s_v[3][PY * PX];    // -vtmp2
  __shared__ R s_p[PY * PX];       // RGAM * pregd at the gradient level
  __shared__ R s_ti[TY * TX], s_tj[TY * TX];
  const TileLv tl = tile_level<VP_DX, VP_DY>(cD.kmin);
  const int l = tl.l, i0 = tl.i0, j0 = tl.j0;
  const int G = cD.G, gmax = cD.G - 2, kmin = cD.kmin;
  const int tid = threadIdx.x, tx = tid % VP_DX, ty = tid / VP_DX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= gmax) && (j <= gmax);
  const R ddc = CC.divdamp_coef;
  const int n = cD.npti;
  const R* cz = CG.C2WGz;
  const R* const* P = a.P.v;
  R gxyz[3] = {R(0.0), R(0.0), R(0.0)};
  int q0 = 0;
  if (own) {
#pragma unroll
    for (int d = 0; d < 3; ++d) gxyz[d] = P2(CG.GRD_x, d, i, j, l);
    q0 = ix(i, j, 0, l);
  }
  {
    const int k = tl.k;
    const int kk = (k == kmin) ? kmin + 1 : k;
    for (int p = tid; p < PX * PY; p += blockDim.x) {
      const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
      R mv[3] = {R(0.0), R(0.0), R(0.0)}, ev[3] = {R(0.0), R(0.0), R(0.0)}, vv[3] = {R(0.0), R(0.0), R(0.0)}, pp = R(0.0);
      if (ii < G && jj < G) {
        const int q = ix(ii, jj, k, l);
        const R rg = CG.RGAM[q], e = a.eth[q];
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const R pv = P[1 + d][q];
          mv[d] = pv * rg;
          ev[d] = (pv * e) * rg;
          vv[d] = -a.vt.f[d][q];
        }
        const int qk = ix(ii, jj, kk, l);
        pp = a.pregd[qk] * CG.RGAM[qk];
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        s_m[d][p] = mv[d];
        s_e[d][p] = ev[d];
        s_v[d][p] = vv[d];
      }
      s_p[p] = pp;
    }
    __syncthreads();
    for (int p = tid; p < TX * TY; p += blockDim.x) {
      const int px = p % TX, py = p / TX;
      const int ii = i0 - 1 + px, jj = j0 - 1 + py;
      R sTI = R(0.0), sTJ = R(0.0);
      if (ii <= G - 2 && jj <= G - 2) {
        const int ia = py * PX + px, ib = ia + 1, ic = ia + PX + 1, id = ia + PX;
        auto C = [&](int dir, int pt, int t) { return P2(CG.coef_intp, (dir * 3 + pt) * 2 + t, ii, jj, l); };
        sTI = C(0, 0, 0) * s_v[0][ia] + C(0, 1, 0) * s_v[0][ib] + C(0, 2, 0) * s_v[0][ic] +
              C(1, 0, 0) * s_v[1][ia] + C(1, 1, 0) * s_v[1][ib] + C(1, 2, 0) * s_v[1][ic] +
              C(2, 0, 0) * s_v[2][ia] + C(2, 1, 0) * s_v[2][ib] + C(2, 2, 0) * s_v[2][ic];
        sTJ = C(0, 0, 1) * s_v[0][ia] + C(0, 1, 1) * s_v[0][ic] + C(0, 2, 1) * s_v[0][id] +
              C(1, 0, 1) * s_v[1][ia] + C(1, 1, 1) * s_v[1][ic] + C(1, 2, 1) * s_v[1][id] +
              C(2, 0, 1) * s_v[2][ia] + C(2, 1, 1) * s_v[2][ic] + C(2, 2, 1) * s_v[2][id];
      }
      s_ti[p] = sTI;
      s_tj[p] = sTJ;
    }
    __syncthreads();
    if (own) {
      const int c0 = (ty + 1) * PX + (tx + 1);
      const int nb[7] = {c0, c0 + 1, c0 + PX + 1, c0 + PX, c0 - 1, c0 - PX - 1, c0 - PX};
      const int q = q0 + (int)k * cD.planei;
      // divergences (div7: per direction left to right, then x + y + z)
      R acc1[3], acc2[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        R s1 = R(0.0), s2 = R(0.0);
#pragma unroll
        for (int m = 0; m < 7; ++m) {
          const R cdv = P2(CG.coef_div, d * 7 + m, i, j, l);
          const R t1 = cdv * s_m[d][nb[m]], t2 = cdv * s_e[d][nb[m]];
          s1 = (m == 0) ? t1 : s1 + t1;
          s2 = (m == 0) ? t2 : s2 + t2;
        }
        acc1[d] = s1;
        acc2[d] = s2;
      }
      h.out[0][q] = acc1[0] + acc1[1] + acc1[2];
      h.out[1][q] = acc2[0] + acc2[1] + acc2[2];
      // 2-D divergence damping, projected
      const int ta = (ty + 1) * TX + (tx + 1);
      const R aTI = s_ti[ta], aTJ = s_tj[ta], bTI = s_ti[ta - 1];
      const R cTI = s_ti[ta - TX - 1], cTJ = s_tj[ta - TX - 1], dTJ = s_tj[ta - TX];
      R dd[3];
#pragma unroll
      for (int d = 0; d < 3; ++d)
        dd[d] = ddc * (P2(CG.coef_diff, d * 6 + 0, i, j, l) * (aTI + aTJ) +
                       P2(CG.coef_diff, d * 6 + 1, i, j, l) * (aTJ + bTI) +
                       P2(CG.coef_diff, d * 6 + 2, i, j, l) * (bTI + cTJ) +
                       P2(CG.coef_diff, d * 6 + 3, i, j, l) * (cTJ + cTI) +
                       P2(CG.coef_diff, d * 6 + 4, i, j, l) * (cTI + dTJ) +
                       P2(CG.coef_diff, d * 6 + 5, i, j, l) * (dTJ + aTI));
      {
        const R prd = div_r(dd[0] * gxyz[0] + dd[1] * gxyz[1] + dd[2] * gxyz[2]);
        dd[0] = dd[0] - div_r(prd * gxyz[0]);
        dd[1] = dd[1] - div_r(prd * gxyz[1]);
        dd[2] = dd[2] - div_r(prd * gxyz[2]);
      }
      // pressure gradient of pregd at level kk
      const int qkk = q0 + (int)kk * cD.planei, qk1 = qkk + cD.planei, qkm = qkk - cD.planei;
      const R P_k1 = a.pregd[qk1], P_k = a.pregd[qkk], P_km = a.pregd[qkm];
      const R rgh1 = CG.RGAMH[qk1], rgh0 = CG.RGAMH[qkk];
      R pg[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        R g = P2(CG.coef_grad, d * 7 + 0, i, j, l) * s_p[nb[0]];
#pragma unroll
        for (int m = 1; m < 7; ++m) g = g + P2(CG.coef_grad, d * 7 + m, i, j, l) * s_p[nb[m]];
        const R up = (cz[(2 * d) * n + qk1] * P_k1 + cz[(2 * d + 1) * n + qk1] * P_k) * rgh1;
        const R dn = (cz[(2 * d) * n + qkk] * P_k + cz[(2 * d + 1) * n + qkk] * P_km) * rgh0;
        pg[d] = g + (up - dn) * CC.rdgz[kk];
      }
      {
        const R prd = div_r(pg[0] * gxyz[0] + pg[1] * gxyz[1] + pg[2] * gxyz[2]);
        pg[0] = pg[0] - div_r(prd * gxyz[0]);
        pg[1] = pg[1] - div_r(prd * gxyz[1]);
        pg[2] = pg[2] - div_r(prd * gxyz[2]);
      }
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        h.out[2 + d][q] = dd[d];
        h.out[5 + d][q] = pg[d];
      }
    }
    __syncthreads();
  }
}

// Column part of vp0 for every regional column: vertical flux convergences,
// small-step tendencies, the implicit matrix and ethtot0, with the horizontal
// terms read from k_vp0_hl (zero on halo columns and outside kmin..kmax, where
// the values that depend on them are replaced by the halo exchanges or the
// boundary rows before they are read).  The column marches upward with every
// half-level quantity evaluated once: at level k the values at k+1 (vertical
// mass and energy fluxes, buoyancy, vertical pressure gradient, gz, pwh,
// half-level eth, the vertical kinetic-energy term) are formed and the ones at
// k and k-1 are carried in registers.  Each value is the expression of
// vp0_column (the pole form), so regional and pole columns round alike.
// 256-thread blocks capped at 64 registers (four per SM; measured faster
// than three at 74 registers)
#define NC_VP0C_BLOCK 256
template <class R>
__global__ void __launch_bounds__(NC_VP0C_BLOCK, NC_MINB(R, 4, NC_F32_VP0C)) k_vp0_cr(Vp0Args<R> a, Vp0H<R> h) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l)) return;
  const Col c = col_reg(i, j, l);
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  const int n = cD.npti;
  const bool in = interior(i, j);
  const R* const* P = a.P.v;
  const double dt = a.dt;
  const double GRAV = cC.GRAV;
  const R* cz = CG.C2WGz;
  const R* c2w = CG.C2W;
  const R* w2c = CG.W2C;
  const double GCVovR = cC.GRAV * cC.CVdry / cC.Rdry;
  const double ACVovRt2 = cC.alpha * cC.CVdry / cC.Rdry / (dt * dt);
  // values at level k (index 0) and k-1 (index m), carried upward
  double vA0 = 0.0, vE0 = 0.0;            // vertical fluxes of rhog / rhoge at half level k
  double gz0 = 0.0, gzm = 0.0;            // gz at k and k-1
  double eh0 = 0.0, ehm = 0.0;            // half-level eth at k and k-1
  double pwh0 = 0.0, dpgw0 = 0.0, dbuo0 = 0.0, vint0 = 0.0;
  for (int k = 0; k < KA; ++k) {
    const int p = c.at(k);
    const int kn = k + 1;
    // ---- half-level values at kn = k+1
    double vA1 = 0.0, vE1 = 0.0, gz1 = 0.0, eh1 = 0.0, pwh1 = 0.0, dpgw1 = 0.0, dbuo1 = 0.0, vint1 = 0.0;
    if (kn < KA) {
      const int q = c.at(kn), qm = c.at(kn - 1);
      if (kn > kmin && kn <= kmax) {
        const double rgh = gam_at(CG.RGAMH, q), rsq = CG.RGSQRTH[q];
        const double z0 = cz[q], z1 = cz[n + q], z2 = cz[2 * n + q], z3 = cz[3 * n + q], z4 = cz[4 * n + q],
                     z5 = cz[5 * n + q];
        const double px = P[1][q], pxm = P[1][qm], py = P[2][q], pym = P[2][qm], pz = P[3][q], pzm = P[3][qm];
        const double e = a.eth[q], em = a.eth[qm], w = P[4][q];
        const double hA = z0 * px + z1 * pxm + z2 * py + z3 * pym + z4 * pz + z5 * pzm;
        vA1 = hA * rgh + 1.0 * w * rsq;
        const double hE = z0 * (px * e) + z1 * (pxm * em) + z2 * (py * e) + z3 * (pym * em) + z4 * (pz * e) +
                          z5 * (pzm * em);
        vE1 = hE * rgh + 1.0 * (w * (cC.afact[kn] * e + cC.bfact[kn] * em)) * rsq;
        // vertical kinetic-energy term of rhogkin
        const double den = c2w[q] * P[0][q] + c2w[n + q] * P[0][qm];
        vint1 = 0.5 * (w * w) / den;
        // buoyancy and vertical pressure gradient
        dbuo1 = -GRAV * (c2w[q] * a.rhogd[q] + c2w[n + q] * a.rhogd[qm]);
        dpgw1 = gam_at(CG.GAM2H, q) * (a.pregd[q] * CG.RGSGAM2[q] - a.pregd[qm] * CG.RGSGAM2[qm]) * cC.rdgzh[kn];
      }
      if (kn >= kmin && kn <= kmax + 1) {
        const int kk = kn;   // kn >= kmin here, so the clamp of rhog_h / eth_h is inactive
        const double rh = c2w[q] * P[0][q] + c2w[n + q] * P[0][c.at(kk - 1)];
        gz1 = GRAV - (dpgw1 - dbuo1) / rh;
        pwh1 = -gz1 * P[4][q];
        eh1 = cC.afact[kk] * a.eth[q] + cC.bfact[kk] * a.eth[c.at(kk - 1)];
      }
    }
    // ---- level k
    const bool hk = in && k >= kmin && k <= kmax;
    const bool kin = k >= kmin && k <= kmax;
    const double div1 = hk ? h.out[0][p] : 0.0, div2 = hk ? h.out[1][p] : 0.0;
    const double drhog = kin ? -div1 - (vA1 - vA0) * cC.rdgz[k] : 0.0;
    const double drhoge = kin ? -div2 - (vE1 - vE0) * cC.rdgz[k] : 0.0;
    double dd[3], dpg[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      dd[d] = hk ? h.out[2 + d][p] : 0.0;
      dpg[d] = hk ? h.out[5 + d][p] : 0.0;
    }
    double pw = 0.0;
    if (kin)
      pw = a.vx[p] * dpg[0] + a.vy[p] * dpg[1] + a.vz[p] * dpg[2] + w2c[p] * pwh1 + w2c[n + p] * pwh0;
    a.gT[0][p] = a.gT0[0][p] + drhog;
    a.gT[1][p] = a.gT0[1][p] - dpg[0] + dd[0] + 0.0;
    a.gT[2][p] = a.gT0[2][p] - dpg[1] + dd[1] + 0.0;
    a.gT[3][p] = a.gT0[3][p] - dpg[2] + dd[2] + 0.0;
    a.gT[4][p] = a.gT0[4][p] + 0.0 * cC.alpha - dpgw0 + dbuo0;
    a.gT[5][p] = a.gT0[5][p] + drhoge + pw;
    if (k >= kmin + 1 && k <= kmax) {
      const int pm = c.at(k - 1), pp = c.at(k + 1);
      const double rg = cC.rdgz[k], rgm = cC.rdgz[k - 1];
      const double Ca = (CG.RGSGAM2[p] * rg + CG.RGSGAM2[pm] * rgm) * gam_at(CG.GAM2H, p);
      const double Cb = cC.dfact[k] - cC.cfact[k - 1];
      const double Cu1 = CG.RGSGAM2[p] * rg * gam_at(CG.GAM2H, pp);
      const double rgh2 = gam_at(CG.RGAMH, p) * gam_at(CG.RGAMH, p);
      const double Cu2 = gam_at(CG.GAM2H, pp) * rgh2 * GCVovR;
      const double Cl1 = CG.RGSGAM2[p] * rg * gam_at(CG.GAM2H, pm);
      const double Cl2 = gam_at(CG.GAM2H, pm) * rgh2 * GCVovR;
      const double rgh = cC.rdgzh[k];
      a.Mc[p] = ACVovRt2 / CG.RGSQRTH[p] + rgh * (Ca * eh0 - Cb * (gz0 + GCVovR));
      a.Mu[p] = -rgh * (Cu1 * eh1 + cC.cfact[k] * (gz1 + Cu2));
      a.Ml[p] = -rgh * (Cl1 * ehm - cC.dfact[k - 1] * (gzm + Cl2));
    }
    double kin0 = 0.0;
    if (kin) {
      const double rg = P[0][p], vx = P[1][p], vy = P[2][p], vz = P[3][p];
      const double kh = 0.5 * (vx * vx + vy * vy + vz * vz) / rg;
      kin0 = kh + w2c[p] * vint1 + w2c[n + p] * vint0;
    }
    a.ethtot0[p] = a.eth[p] + kin0 / P[0][p] + CG.PHI[p];
    vA0 = vA1; vE0 = vE1;
    gzm = gz0; gz0 = gz1;
    ehm = eh0; eh0 = eh1;
    pwh0 = pwh1; dpgw0 = dpgw1; dbuo0 = dbuo1; vint0 = vint1;
  }
}

template <class R>
__global__ void k_vp0(Vp0Args<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  if (!pole) vp0_column<R, false>(a, i, j, l, 0, 0);
  else vp0_column<R, true>(a, 0, 0, 0, g, lp);
}

// ---------------------------------------------------------------------------
// acoustic loop, path1 (kernels/vipath1.py:68-160): diff_vh with BNDCND and
// the running mean of the horizontal momentum.
// ---------------------------------------------------------------------------
template <class R>
struct Path1Args {
  const R* PS[6];     // PROG_split (RHOGE boundary rows read clamped)
  const R* rhog;      // PROG rhog
  const R* gT[6];
  CThree<R> vt;               // post-COMM 3-D divdamp of PROG_split
  R* dvh[3];          // out
  R* PM[5];           // running mean (in/out)
  R dt, rweight, RovCV;
};

template <class R, bool POLE>
__device__ void path1_column(const Path1Args<R>& a, int i, int j, int l, int g, int lp) {
  const Col c = POLE ? col_pl(g, lp) : col_reg(i, j, l);
  const MetT<R> m = met_of<R>(POLE);
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  const R dt = a.dt;
  auto pregs = [&](int base_q, int kk) -> R {  // preg_prim_split with clamped boundary rows
    int k2 = kk < kmin ? kmin : (kk > kmax ? kmax : kk);
    return a.PS[5][base_q + (int)k2 * c.ks] * a.RovCV;
  };
  R vals[3][2];  // values at kmin and kmax for the boundary rows
  R* const* out = a.dvh;
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    R dd[3], pg[3];
    if (!POLE) {
      divdamp2d_at(a.vt, i, j, k, l, dd);
      presgrad_reg(i, j, k, l, c, m, [&](int ii, int jj, int kk) { return pregs(ix(ii, jj, 0, l), kk); }, pg);
    } else {
      divdamp2d_pl_at(a.vt, g, k, lp, dd);
      presgrad_pl(g, k, lp, c, m, [&](int gg, int kk) { return pregs((int)gg * cD.KA * cD.LP + lp, kk); }, pg);
    }
    for (int d = 0; d < 3; ++d) {
      R drv = a.gT[1 + d][p] - pg[d] + dd[d] + R(0.0);
      R v = a.PS[1 + d][p] + drv * dt;
      out[d][p] = v;
      if (k == kmin) vals[d][0] = v;
      if (k == kmax) vals[d][1] = v;
    }
  }
  const int pT = c.at(kmax + 1), pK = c.at(kmax), pB = c.at(kmin - 1), pN = c.at(kmin);
  for (int d = 0; d < 3; ++d) {
    out[d][pT] = R(1.0) * (vals[d][1] / a.rhog[pK]) * a.rhog[pT];
    out[d][pB] = -R(1.0) * (vals[d][0] / a.rhog[pN]) * a.rhog[pB];
  }
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    for (int d = 0; d < 3; ++d) a.PM[1 + d][p] = a.PM[1 + d][p] + out[d][p] * a.rweight;
  }
}

// Regional path 1, one block per (level, tile): same stencils and
// arithmetic as path1_column.  The blocks at kmin and kmax also write the
// boundary rows kmin-1 and kmax+1 from the values they computed.
template <class R>
__global__ void __launch_bounds__(DD_DX * DD_DY, DD_MINB(NC_MINB(R, 6, NC_F32_PATH1))) k_path1_l(Path1Args<R> a) {
  constexpr int PX = DD_DX + 2, PY = DD_DY + 2, TX = DD_DX + 1, TY = DD_DY + 1;
  __shared__ R s_v[3][PY * PX];
  __shared__ R s_p[PY * PX];
  __shared__ R s_ti[TY * TX], s_tj[TY * TX];
  const TileLv tl = tile_level<DD_DX, DD_DY>(cD.kmin);
  const int k = tl.k, l = tl.l, i0 = tl.i0, j0 = tl.j0;
  const int G = cD.G, gmax = cD.G - 2, kmin = cD.kmin, kmax = cD.kmax;
  const int kk = (k == kmin) ? kmin + 1 : k;
  const int tid = threadIdx.x, tx = tid % DD_DX, ty = tid / DD_DX;
  const R RovCV = a.RovCV;
  for (int p = tid; p < PX * PY; p += blockDim.x) {
    const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
    R x = R(0.0), y = R(0.0), z = R(0.0), pp = R(0.0);
    if (ii < G && jj < G) {
      const int q = ix(ii, jj, k, l);
      x = -__ldg(&a.vt.f[0][q]);
      y = -__ldg(&a.vt.f[1][q]);
      z = -__ldg(&a.vt.f[2][q]);
      const int qk = ix(ii, jj, kk, l);
      pp = __ldg(&a.PS[5][qk]) * RovCV * __ldg(&CG.RGAM[qk]);
    }
    s_v[0][p] = x;
    s_v[1][p] = y;
    s_v[2][p] = z;
    s_p[p] = pp;
  }
  __syncthreads();
  for (int p = tid; p < TX * TY; p += blockDim.x) {
    const int px = p % TX, py = p / TX;
    const int ii = i0 - 1 + px, jj = j0 - 1 + py;
    R sTI = R(0.0), sTJ = R(0.0);
    if (ii <= G - 2 && jj <= G - 2) {
      const int ia = py * PX + px, ib = ia + 1, ic = ia + PX + 1, id = ia + PX;
      auto C = [&](int dir, int pt, int t) { return P2c(CG.coef_intp, (dir * 3 + pt) * 2 + t, ii, jj, l); };
      sTI = C(0, 0, 0) * s_v[0][ia] + C(0, 1, 0) * s_v[0][ib] + C(0, 2, 0) * s_v[0][ic] +
            C(1, 0, 0) * s_v[1][ia] + C(1, 1, 0) * s_v[1][ib] + C(1, 2, 0) * s_v[1][ic] +
            C(2, 0, 0) * s_v[2][ia] + C(2, 1, 0) * s_v[2][ib] + C(2, 2, 0) * s_v[2][ic];
      sTJ = C(0, 0, 1) * s_v[0][ia] + C(0, 1, 1) * s_v[0][ic] + C(0, 2, 1) * s_v[0][id] +
            C(1, 0, 1) * s_v[1][ia] + C(1, 1, 1) * s_v[1][ic] + C(1, 2, 1) * s_v[1][id] +
            C(2, 0, 1) * s_v[2][ia] + C(2, 1, 1) * s_v[2][ic] + C(2, 2, 1) * s_v[2][id];
    }
    s_ti[p] = sTI;
    s_tj[p] = sTJ;
  }
  __syncthreads();
  const int i = i0 + tx, j = j0 + ty;
  if (i > gmax || j > gmax) return;
  const R ddc = CC.divdamp_coef, dt = a.dt, rweight = a.rweight;
  const int n = cD.npti;
  const R* cz = CG.C2WGz;
  const R gx = P2c(CG.GRD_x, 0, i, j, l), gy = P2c(CG.GRD_x, 1, i, j, l), gz = P2c(CG.GRD_x, 2, i, j, l);
  const int q0 = ix(i, j, 0, l);
  auto Pown = [&](int k2) {
    const int kc = k2 < kmin ? kmin : (k2 > kmax ? kmax : k2);
    return __ldg(&a.PS[5][q0 + (int)kc * cD.planei]) * RovCV;
  };
  const int ta = (ty + 1) * TX + (tx + 1);
  const R aTI = s_ti[ta], aTJ = s_tj[ta], bTI = s_ti[ta - 1];
  const R cTI = s_ti[ta - TX - 1], cTJ = s_tj[ta - TX - 1], dTJ = s_tj[ta - TX];
  R dd[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
    dd[d] = ddc * (P2c(CG.coef_diff, d * 6 + 0, i, j, l) * (aTI + aTJ) + P2c(CG.coef_diff, d * 6 + 1, i, j, l) * (aTJ + bTI) +
                   P2c(CG.coef_diff, d * 6 + 2, i, j, l) * (bTI + cTJ) + P2c(CG.coef_diff, d * 6 + 3, i, j, l) * (cTJ + cTI) +
                   P2c(CG.coef_diff, d * 6 + 4, i, j, l) * (cTI + dTJ) + P2c(CG.coef_diff, d * 6 + 5, i, j, l) * (dTJ + aTI));
  {
    const R prd = div_r(dd[0] * gx + dd[1] * gy + dd[2] * gz);
    dd[0] = dd[0] - div_r(prd * gx);
    dd[1] = dd[1] - div_r(prd * gy);
    dd[2] = dd[2] - div_r(prd * gz);
  }
  const int c0 = (ty + 1) * PX + (tx + 1);
  const R s7[7] = {s_p[c0], s_p[c0 + 1], s_p[c0 + PX + 1], s_p[c0 + PX], s_p[c0 - 1], s_p[c0 - PX - 1], s_p[c0 - PX]};
  const int qkk = q0 + (int)kk * cD.planei, qk1 = qkk + cD.planei;
  const R P_k1 = Pown(kk + 1), P_k = Pown(kk), P_km = Pown(kk - 1);
  const R rgh1 = __ldg(&CG.RGAMH[qk1]), rgh0 = __ldg(&CG.RGAMH[qkk]);
  R pg[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    R g = P2c(CG.coef_grad, d * 7 + 0, i, j, l) * s7[0];
#pragma unroll
    for (int m = 1; m < 7; ++m) g = g + P2c(CG.coef_grad, d * 7 + m, i, j, l) * s7[m];
    const R up = (__ldg(&cz[(2 * d) * n + qk1]) * P_k1 + __ldg(&cz[(2 * d + 1) * n + qk1]) * P_k) * rgh1;
    const R dn = (__ldg(&cz[(2 * d) * n + qkk]) * P_k + __ldg(&cz[(2 * d + 1) * n + qkk]) * P_km) * rgh0;
    pg[d] = g + (up - dn) * CC.rdgz[kk];
  }
  {
    const R prd = div_r(pg[0] * gx + pg[1] * gy + pg[2] * gz);
    pg[0] = pg[0] - div_r(prd * gx);
    pg[1] = pg[1] - div_r(prd * gy);
    pg[2] = pg[2] - div_r(prd * gz);
  }
  const int q = q0 + (int)k * cD.planei;
  R v[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const R drv = __ldg(&a.gT[1 + d][q]) - pg[d] + dd[d] + R(0.0);
    v[d] = __ldg(&a.PS[1 + d][q]) + drv * dt;
    a.dvh[d][q] = v[d];
    a.PM[1 + d][q] = a.PM[1 + d][q] + v[d] * rweight;
  }
  if (k == kmin) {
    const int pB = q - cD.planei;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const R vB = -R(1.0) * (v[d] / __ldg(&a.rhog[q])) * __ldg(&a.rhog[pB]);
      a.dvh[d][pB] = vB;
      a.PM[1 + d][pB] = a.PM[1 + d][pB] + vB * rweight;
    }
  }
  if (k == kmax) {
    const int pT = q + cD.planei;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const R vT = R(1.0) * (v[d] / __ldg(&a.rhog[q])) * __ldg(&a.rhog[pT]);
      a.dvh[d][pT] = vT;
      a.PM[1 + d][pT] = a.PM[1 + d][pT] + vT * rweight;
    }
  }
}

template <class R>
__global__ void k_path1(Path1Args<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  if (!pole) path1_column<R, false>(a, i, j, l, 0, 0);
  else path1_column<R, true>(a, 0, 0, 0, g, lp);
}

// ---------------------------------------------------------------------------
// vi_main (kernels/vimain.py:127-262): horizontal divergences (kernel A),
// then per column the flux convergences, the tridiagonal Thomas solve
// (kernels/virhowsolver.py:42-120), kinetic energies and the energy update.
// ---------------------------------------------------------------------------
template <class R>
struct VimainArgs {
  const R* PS[6];
  const R* P[6];          // PROG
  const R *eth, *ethtot0;
  const R* gT[6];         // small-step tendency
  const R* gT0e;          // large-step tendency of RHOGE (grhogetot)
  const double *Mc, *Mu, *Ml;  // float64 in both forms
  CThree<R> dvh;                  // post-COMM diff_vh
  R* hdiv[3];             // kernel A output
  R* dwe[3];              // out: rhog_s1, rhogw_s1, rhoge_s1
  R* PM0;                 // running mean of RHOG (in/out)
  R* PM4;                 // running mean of RHOGW (in/out)
  double dt, rweight, RovCV;
};

template <class R>
__global__ void k_vimain_a(VimainArgs<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!pole) {
    if (!col_of(t, i, j, l)) return;
    const bool in = interior(i, j);
    for (int k = 0; k < cD.KA; ++k) {
      int p = ix(i, j, k, l);
      R h1 = R(0.0), h2 = R(0.0), h3 = R(0.0);
      if (in && k >= cD.kmin && k <= cD.kmax) {
        h1 = div7<R>(i, j, k, l, [&](int ii, int jj, int kk, int d) {
          int q = ix(ii, jj, kk, l);
          return a.dvh.f[d][q] * gam_at(CG.RGAM, q);
        });
        h2 = div7<R>(i, j, k, l, [&](int ii, int jj, int kk, int d) {
          int q = ix(ii, jj, kk, l);
          return (a.dvh.f[d][q] * a.eth[q]) * gam_at(CG.RGAM, q);
        });
        h3 = div7<R>(i, j, k, l, [&](int ii, int jj, int kk, int d) {
          int q = ix(ii, jj, kk, l);
          return ((a.P[1 + d][q] + a.dvh.f[d][q]) * a.ethtot0[q]) * gam_at(CG.RGAM, q);
        });
      }
      a.hdiv[0][p] = h1; a.hdiv[1][p] = h2; a.hdiv[2][p] = h3;
    }
  } else {
    int tp = t;
    if (tp < cD.KA * cD.LP) {
      int k = (int)(tp / cD.LP), lp = (int)(tp % cD.LP);
      for (int g = 0; g < 6; ++g) {
        int p = ipl(g, k, lp);
        R h1 = R(0.0), h2 = R(0.0), h3 = R(0.0);
        if (g == 0 && k >= cD.kmin && k <= cD.kmax) {
          h1 = div_pl<R>(lp, k, [&](int q, int d) { return a.dvh.f[d][q]; });
          h2 = div_pl<R>(lp, k, [&](int q, int d) { return a.dvh.f[d][q] * a.eth[q]; });
          h3 = div_pl<R>(lp, k, [&](int q, int d) { return (a.P[1 + d][q] + a.dvh.f[d][q]) * a.ethtot0[q]; });
        }
        a.hdiv[0][p] = h1; a.hdiv[1][p] = h2; a.hdiv[2][p] = h3;
      }
    }
  }
}

// vi_main kernel A, one block per (level, tile): the horizontal divergences
// of RGAM*diff_vh, RGAM*diff_vh*eth and RGAM*(rhogv + diff_vh)*ethtot0.
template <class R>
__global__ void __launch_bounds__(DD_DX * DD_DY, DD_MINB(NC_MINB(R, 6, NC_F32_VIMAINA))) k_vimain_a_l(VimainArgs<R> a) {
  constexpr int PX = DD_DX + 2, PY = DD_DY + 2;
  __shared__ R s_h[3][3][PY * PX];
  const TileLv tl = tile_level<DD_DX, DD_DY>(cD.kmin);
  const int l = tl.l, i0 = tl.i0, j0 = tl.j0;
  const int G = cD.G, gmax = cD.G - 2;
  const int tid = threadIdx.x, tx = tid % DD_DX, ty = tid / DD_DX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= gmax) && (j <= gmax);
  {
    const int k = tl.k;
    for (int p = tid; p < PX * PY; p += blockDim.x) {
      const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
      if (ii < G && jj < G) {
        const int q = ix(ii, jj, k, l);
        const R rg = gam_at_ldg(CG.RGAM, q), e = __ldg(&a.eth[q]), et = __ldg(&a.ethtot0[q]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const R dv = __ldg(&a.dvh.f[d][q]);
          s_h[0][d][p] = dv * rg;
          s_h[1][d][p] = (dv * e) * rg;
          s_h[2][d][p] = ((__ldg(&a.P[1 + d][q]) + dv) * et) * rg;
        }
      } else {
#pragma unroll
        for (int f = 0; f < 3; ++f)
#pragma unroll
          for (int d = 0; d < 3; ++d) s_h[f][d][p] = R(0.0);
      }
    }
    __syncthreads();
    if (own) {
      const int c0 = (ty + 1) * PX + (tx + 1);
      const int nb[7] = {c0, c0 + 1, c0 + PX + 1, c0 + PX, c0 - 1, c0 - PX - 1, c0 - PX};
      const int q = ix(i, j, k, l);
      R acc[3][3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        R s[3] = {R(0.0), R(0.0), R(0.0)};
#pragma unroll
        for (int m = 0; m < 7; ++m) {
          const R cdv = P2c(CG.coef_div, d * 7 + m, i, j, l);
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            const R t = cdv * s_h[f][d][nb[m]];
            s[f] = (m == 0) ? t : s[f] + t;
          }
        }
#pragma unroll
        for (int f = 0; f < 3; ++f) acc[f][d] = s[f];
      }
#pragma unroll
      for (int f = 0; f < 3; ++f) a.hdiv[f][q] = acc[f][0] + acc[f][1] + acc[f][2];
    }
    __syncthreads();
  }
}

// vi_main A with VA_NK levels per block: the cell's divergence coefficients
// (coef_div, 21 planes) are held in registers once for all of the block's
// levels instead of re-read from L2 at every level.  Same expressions in the
// same order as k_vimain_a_l (same results).  Used by the float instance
// (gl08: 6.0 -> 5.5 ms per step); the double one stays on k_vimain_a_l, which
// is faster there (9.9 against 11.6 ms: 42 more registers cost residency).
#ifndef VA_NK
#define VA_NK 5
#endif
template <class R>
__global__ void __launch_bounds__(DD_DX * DD_DY, DD_MINB(NC_MINB(R, 4, 5))) k_vimain_a_m(VimainArgs<R> a) {
  constexpr int PX = DD_DX + 2, PY = DD_DY + 2;
  __shared__ R s_h[3][3][PY * PX];
  const int ntx = (cD.G - 2 + DD_DX - 1) / DD_DX;
  const int l = (int)blockIdx.z;
  const int i0 = 1 + ((int)blockIdx.y % ntx) * DD_DX, j0 = 1 + ((int)blockIdx.y / ntx) * DD_DY;
  const int ka = cD.kmin + (int)blockIdx.x * VA_NK, kb = min(ka + VA_NK - 1, cD.kmax);
  const int G = cD.G, gmax = cD.G - 2;
  const int tid = threadIdx.x, tx = tid % DD_DX, ty = tid / DD_DX;
  const int i = i0 + tx, j = j0 + ty;
  const bool own = (i <= gmax) && (j <= gmax);
  R cdv[21];
  if (own) {
#pragma unroll
    for (int m = 0; m < 21; ++m) cdv[m] = P2c(CG.coef_div, m, i, j, l);
  }
  for (int k = ka; k <= kb; ++k) {
    for (int p = tid; p < PX * PY; p += blockDim.x) {
      const int ii = i0 - 1 + p % PX, jj = j0 - 1 + p / PX;
      if (ii < G && jj < G) {
        const int q = ix(ii, jj, k, l);
        const R rg = gam_at_ldg(CG.RGAM, q), e = __ldg(&a.eth[q]), et = __ldg(&a.ethtot0[q]);
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const R dv = __ldg(&a.dvh.f[d][q]);
          s_h[0][d][p] = dv * rg;
          s_h[1][d][p] = (dv * e) * rg;
          s_h[2][d][p] = ((__ldg(&a.P[1 + d][q]) + dv) * et) * rg;
        }
      } else {
#pragma unroll
        for (int f = 0; f < 3; ++f)
#pragma unroll
          for (int d = 0; d < 3; ++d) s_h[f][d][p] = R(0.0);
      }
    }
    __syncthreads();
    if (own) {
      const int c0 = (ty + 1) * PX + (tx + 1);
      const int nb[7] = {c0, c0 + 1, c0 + PX + 1, c0 + PX, c0 - 1, c0 - PX - 1, c0 - PX};
      const int q = ix(i, j, k, l);
      R acc[3][3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        R sv[3] = {R(0.0), R(0.0), R(0.0)};
#pragma unroll
        for (int m = 0; m < 7; ++m) {
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            const R t = cdv[d * 7 + m] * s_h[f][d][nb[m]];
            sv[f] = (m == 0) ? t : sv[f] + t;
          }
        }
#pragma unroll
        for (int f = 0; f < 3; ++f) acc[f][d] = sv[f];
      }
#pragma unroll
      for (int f = 0; f < 3; ++f) a.hdiv[f][q] = acc[f][0] + acc[f][1] + acc[f][2];
    }
    __syncthreads();
  }
}

// One pole column of vi_main.  In the mixed form the flux convergences and
// the energy update run in float32 (R) and the tridiagonal solve in float64,
// as in the regional kernels k_vi_solve / k_vi_energy_p.
template <class R, bool POLE>
__device__ void vimain_column(const VimainArgs<R>& a, const Col c) {
  const MetT<R> m = met_of<R>(POLE);
  const int KA = cD.KA, kmin = cD.kmin, kmax = cD.kmax;
  const double dt = a.dt;
  const R dtR = R(a.dt);
  const double Rdry = cC.Rdry, CVdry = cC.CVdry;
  auto PSk = [&](int comp, int k) -> R {  // PROG_split with clamped RHOGE boundary rows
    if (comp == 5) k = k < kmin ? kmin : (k > kmax ? kmax : k);
    return a.PS[comp][c.at(k)];
  };
  auto preg0 = [&](int k) -> double { return (double)PSk(5, k) * a.RovCV; };
  auto DV = [&](int k, int d) -> R { return a.dvh.f[d][c.at(k)]; };
  auto DVE = [&](int k, int d) -> R { return a.dvh.f[d][c.at(k)] * a.eth[c.at(k)]; };
  // grhog1 and gpre on every level
  double grhog1[NC_MAXK], gpre[NC_MAXK];
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    R drhog = fluxconv_col(c, m, k, a.hdiv[0][p], R(0.0), DV, [&](int kk) { return PSk(4, kk); });
    R drhoge = fluxconv_col(c, m, k, a.hdiv[1][p], R(0.0), DVE, [&](int kk) { return R(0.0); });
    grhog1[k] = (double)a.gT[0][p] + (double)drhog;
    double grhoge1 = (double)a.gT[5][p] + (double)drhoge;
    gpre[k] = grhoge1 * Rdry / CVdry;
  }
  // Thomas solve (kernels/virhowsolver.py:67-120), float64
  const int kT = kmax + 1;
  double rw_top = -((double)mc(m.C2WGz, c, 0, 6, kT) * DV(kT, 0) + (double)mc(m.C2WGz, c, 1, 6, kT) * DV(kmax, 0) +
                    (double)mc(m.C2WGz, c, 2, 6, kT) * DV(kT, 1) + (double)mc(m.C2WGz, c, 3, 6, kT) * DV(kmax, 1) +
                    (double)mc(m.C2WGz, c, 4, 6, kT) * DV(kT, 2) + (double)mc(m.C2WGz, c, 5, 6, kT) * DV(kmax, 2));
  const double CVovRt2 = CVdry / Rdry / (dt * dt);
  const double rw_kmin = 0.0 * (double)m.RGSGAM2H[c.at(kmin)];
  const double rw_kmaxp1 = rw_top * (double)m.RGSGAM2H[c.at(kT)];
  const int N = kmax - kmin;
  double u[NC_MAXK], gam[NC_MAXK];
  double beta = 0.0;
  for (int n = 0; n < N; ++n) {
    int k = kmin + 1 + n;
    int p = c.at(k), pm = c.at(k - 1);
    double rg2 = (double)gam_at(m.RGAMH, p) * (double)gam_at(m.RGAMH, p);
    double rgam2 = (double)gam_at(m.RGAM, p) * (double)gam_at(m.RGAM, p);
    double rgam2m = (double)gam_at(m.RGAM, pm) * (double)gam_at(m.RGAM, pm);
    double Sw = (double)a.gT[4][p] + 0.0 * cC.alpha;
    double S = (((double)PSk(4, k) * cC.alpha + dt * Sw) * rg2 -
                ((preg0(k) + dt * gpre[k]) * (double)m.RGSGAM2[p] - (preg0(k - 1) + dt * gpre[k - 1]) * (double)m.RGSGAM2[pm]) *
                    dt * cC.rdgzh[k] -
                (((double)PSk(0, k) + dt * grhog1[k]) * rgam2 * cC.afact[k] +
                 ((double)PSk(0, k - 1) + dt * grhog1[k - 1]) * rgam2m * cC.bfact[k]) *
                    dt * cC.GRAV) *
               CVovRt2;
    if (n == 0) S = S - a.Ml[c.at(kmin + 1)] * rw_kmin;
    if (n == N - 1) S = S - a.Mu[c.at(kmax)] * rw_kmaxp1;
    double Mc = a.Mc[p], Ml = a.Ml[p];
    if (n == 0) {
      beta = Mc;
      u[0] = S / beta;
    } else {
      double gg = a.Mu[pm] / beta;
      beta = Mc - Ml * gg;
      u[n] = (S - Ml * u[n - 1]) / beta;
      gam[n] = gg;
    }
  }
  R rws1[NC_MAXK];
  for (int k = 0; k < KA; ++k) rws1[k] = R(0.0);
  {
    double x = u[N - 1];
    rws1[kmin + N] = R(x * (double)m.GSGAM2H[c.at(kmin + N)]);
    for (int n = N - 2; n >= 0; --n) {
      x = u[n] - gam[n + 1] * x;
      rws1[kmin + 1 + n] = R(x * (double)m.GSGAM2H[c.at(kmin + 1 + n)]);
    }
    rws1[kmin] = R(rw_kmin * (double)m.GSGAM2H[c.at(kmin)]);
    rws1[kT] = R(rw_kmaxp1 * (double)m.GSGAM2H[c.at(kT)]);
  }
  // rhog_split1, kinetic energies, total-energy advection, rhoge_split1
  R rs1[NC_MAXK];
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    R drhog2 = fluxconv_col(c, m, k, a.hdiv[0][p], R(1.0), DV, [&](int kk) { return rws1[kk]; });
    rs1[k] = PSk(0, k) + (a.gT[0][p] + drhog2) * dtR;
  }
  for (int k = 0; k < KA; ++k) {
    int p = c.at(k);
    auto st10 = [&](int kk, int comp) -> R {
      int q = c.at(kk);
      return a.P[comp][q] + PSk(comp, kk);
    };
    auto st11 = [&](int kk, int comp) -> R {
      int q = c.at(kk);
      if (comp == 0) return a.P[0][q] + rs1[kk];
      if (comp == 4) return a.P[4][q] + rws1[kk];
      return a.P[comp][q] + a.dvh.f[comp - 1][q];
    };
    R kin10 = rhogkin_at(c, m, k, st10);
    R kin11 = rhogkin_at(c, m, k, st11);
    R drhogetot = fluxconv_col(
        c, m, k, a.hdiv[2][p], R(1.0),
        [&](int kk, int d) {
          int q = c.at(kk);
          return (a.P[1 + d][q] + a.dvh.f[d][q]) * a.ethtot0[q];
        },
        [&](int kk) {
          int q = c.at(kk), qm = c.at(kk - 1);
          return (a.P[4][q] + rws1[kk]) * (CC.afact[kk] * a.ethtot0[q] + CC.bfact[kk] * a.ethtot0[qm]);
        });
    R re = PSk(5, k) + (a.gT0e[p] + drhogetot) * dtR + (kin10 - kin11) + (PSk(0, k) - rs1[k]) * m.PHI[p];
    a.dwe[0][p] = rs1[k];
    a.dwe[1][p] = rws1[k];
    a.dwe[2][p] = re;
    a.PM0[p] = a.PM0[p] + rs1[k] * R(a.rweight);
    a.PM4[p] = a.PM4[p] + rws1[k] * R(a.rweight);
  }
}

// Regional vi_main in two column kernels (interior columns; the halo columns
// of the outputs are replaced by the exchange that follows).
// k_vi_solve: flux convergences of diff_vh (rolling half-level fluxes), the
// Thomas forward sweep, then the back substitution fused with rhog_split1 on
// the way down; writes rhog_s1, rhogw_s1 and their running means.
// nine 128-thread blocks per SM (56 registers): the 655,360 interior columns
// of gl08 fill 3.84 waves of the 148 SMs instead of 4.32 at eight
// GU: the gamma factors are all 1 and are not loaded; the other instance loads them
template <class R, bool GU>
__global__ void __launch_bounds__(128, NC_MINB(R, 9, NC_F32_VISOLVE)) k_vi_solve(VimainArgs<R> a) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l;
  if (!col_of(t, i, j, l) || !interior(i, j)) return;
  const Col c = col_reg(i, j, l);
  const MetT<R> m = met_of<R>(false);
  const int kmin = cD.kmin, kmax = cD.kmax, kT = kmax + 1;
  const double dt = a.dt, Rdry = cC.Rdry, CVdry = cC.CVdry, RovCV = a.RovCV;
  const int n = cD.npti;
  const R* cz = CG.C2WGz;
  const R* const* DVp = a.dvh.f;
  auto preg0 = [&](int k) -> double {
    const int k2 = k < kmin ? kmin : (k > kmax ? kmax : k);
    return a.PS[5][c.at(k2)] * RovCV;
  };
  // horizontal part of the half-level flux of diff_vh (and of diff_vh*eth) at kk
  auto hflux = [&](int kk, bool withe) -> double {
    const int q = c.at(kk), qm = c.at(kk - 1);
    const double e = withe ? a.eth[q] : 1.0, em = withe ? a.eth[qm] : 1.0;
    double f0 = DVp[0][q], f0m = DVp[0][qm], f1 = DVp[1][q], f1m = DVp[1][qm], f2 = DVp[2][q], f2m = DVp[2][qm];
    if (withe) {
      f0 = f0 * e; f0m = f0m * em; f1 = f1 * e; f1m = f1m * em; f2 = f2 * e; f2m = f2m * em;
    }
    const double h = cz[q] * f0 + cz[n + q] * f0m + cz[2 * n + q] * f1 + cz[3 * n + q] * f1m + cz[4 * n + q] * f2 +
                     cz[5 * n + q] * f2m;
    return h * (GU ? 1.0 : m.RGAMH[q]);
  };
  double hD[NC_MAXK];
  const int pT = c.at(kT), pK = c.at(kmax);
  const double rw_top = -(cz[pT] * DVp[0][pT] + cz[n + pT] * DVp[0][pK] + cz[2 * n + pT] * DVp[1][pT] +
                          cz[3 * n + pT] * DVp[1][pK] + cz[4 * n + pT] * DVp[2][pT] + cz[5 * n + pT] * DVp[2][pK]);
  const double CVovRt2 = CVdry / Rdry / (dt * dt);
  const double rw_kmin = 0.0 * m.RGSGAM2H[c.at(kmin)];
  const double rw_kmaxp1 = rw_top * m.RGSGAM2H[pT];
  const int N = kmax - kmin;
  double u[NC_MAXK], gam[NC_MAXK];
  double vD_lo = 0.0, vE_lo = 0.0, g1_prev = 0.0, gp_prev = 0.0, beta = 0.0;
  for (int k = kmin; k <= kmax; ++k) {
    const int p = c.at(k);
    const int kk = k + 1;
    double vD_hi = 0.0, vE_hi = 0.0;
    if (kk <= kmax) {
      const double hd = hflux(kk, false);
      hD[kk] = hd;
      const double rq = m.RGSQRTH[c.at(kk)];
      vD_hi = hd + 0.0 * a.PS[4][c.at(kk)] * rq;
      vE_hi = hflux(kk, true) + 0.0 * 0.0 * rq;
    }
    const double drhog = -a.hdiv[0][p] - (vD_hi - vD_lo) * cC.rdgz[k];
    const double drhoge = -a.hdiv[1][p] - (vE_hi - vE_lo) * cC.rdgz[k];
    const double g1 = a.gT[0][p] + drhog;
    const double gp = (a.gT[5][p] + drhoge) * Rdry / CVdry;
    if (k >= kmin + 1) {
      const int nn = k - kmin - 1;
      const int pm = c.at(k - 1);
      const double rgh = GU ? 1.0 : m.RGAMH[p], rgm = GU ? 1.0 : m.RGAM[p], rgmm = GU ? 1.0 : m.RGAM[pm];
      const double rg2 = rgh * rgh;
      const double rgam2 = rgm * rgm, rgam2m = rgmm * rgmm;
      const double Sw = a.gT[4][p] + 0.0 * cC.alpha;
      double S = ((a.PS[4][p] * cC.alpha + dt * Sw) * rg2 -
                  ((preg0(k) + dt * gp) * m.RGSGAM2[p] - (preg0(k - 1) + dt * gp_prev) * m.RGSGAM2[pm]) * dt *
                      cC.rdgzh[k] -
                  ((a.PS[0][p] + dt * g1) * rgam2 * cC.afact[k] + (a.PS[0][pm] + dt * g1_prev) * rgam2m * cC.bfact[k]) *
                      dt * cC.GRAV) *
                 CVovRt2;
      if (nn == 0) S = S - a.Ml[c.at(kmin + 1)] * rw_kmin;
      if (nn == N - 1) S = S - a.Mu[c.at(kmax)] * rw_kmaxp1;
      const double Mc = a.Mc[p], Ml = a.Ml[p];
      if (nn == 0) {
        beta = Mc;
        u[0] = S / beta;
      } else {
        const double gg = a.Mu[pm] / beta;
        beta = Mc - Ml * gg;
        u[nn] = (S - Ml * u[nn - 1]) / beta;
        gam[nn] = gg;
      }
    }
    g1_prev = g1;
    gp_prev = gp;
    vD_lo = vD_hi;
    vE_lo = vE_hi;
  }
  // back substitution (downward) fused with rhog_split1
  double x = 0.0, v2_hi = 0.0;
  for (int k = kT; k >= 0; --k) {
    const int p = c.at(k);
    double rws;
    if (k == kT) {
      rws = rw_kmaxp1 * m.GSGAM2H[p];
    } else if (k >= kmin + 1) {
      const int nn = k - kmin - 1;
      x = (nn == N - 1) ? u[N - 1] : u[nn] - gam[nn + 1] * x;
      rws = x * m.GSGAM2H[p];
    } else if (k == kmin) {
      rws = rw_kmin * m.GSGAM2H[p];
    } else {
      rws = 0.0;
    }
    const double v2 = (k > kmin && k <= kmax) ? hD[k] + 1.0 * rws * m.RGSQRTH[p] : 0.0;
    double drhog2 = 0.0;
    if (k >= kmin && k <= kmax) drhog2 = -a.hdiv[0][p] - (v2_hi - v2) * cC.rdgz[k];
    const double rs = a.PS[0][p] + (a.gT[0][p] + drhog2) * dt;
    a.dwe[0][p] = rs;
    a.dwe[1][p] = rws;
    a.PM0[p] = a.PM0[p] + rs * a.rweight;
    a.PM4[p] = a.PM4[p] + rws * a.rweight;
    v2_hi = v2;
  }
}

// vi_main energy update with one thread per interior grid point: kinetic
// energies, total-energy advection and rhoge_split1 from the rhog_s1 /
// rhogw_s1 written by k_vi_solve (no vertical recurrence; neighbouring levels
// are read through the cache).
template <class R>
__global__ void __launch_bounds__(128, NC_MINB(R, 1, NC_F32_VIENERGY)) k_vi_energy_p(VimainArgs<R> a) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= cD.npti) return;
  const int G = cD.G, KA = cD.KA;
  const int i = (int)(t % G), j = (int)((t / G) % G), k = (int)((t / ((int)G * G)) % KA);
  const int l = (int)(t / ((int)G * G * KA));
  if (!interior(i, j)) return;
  const Col c = col_reg(i, j, l);
  const MetT<R> m = met_of<R>(false);
  const int kmin = cD.kmin, kmax = cD.kmax;
  const R* rs1 = a.dwe[0];
  const R* rws1 = a.dwe[1];
  auto PSk = [&](int comp, int kk) -> R {
    if (comp == 5) kk = kk < kmin ? kmin : (kk > kmax ? kmax : kk);
    return a.PS[comp][c.at(kk)];
  };
  const int p = c.at(k);
  auto st10 = [&](int kk, int comp) -> R { return a.P[comp][c.at(kk)] + PSk(comp, kk); };
  auto st11 = [&](int kk, int comp) -> R {
    const int q = c.at(kk);
    if (comp == 0) return a.P[0][q] + rs1[q];
    if (comp == 4) return a.P[4][q] + rws1[q];
    return a.P[comp][q] + a.dvh.f[comp - 1][q];
  };
  const R kin10 = rhogkin_at(c, m, k, st10);
  const R kin11 = rhogkin_at(c, m, k, st11);
  const R drhogetot = fluxconv_col(
      c, m, k, a.hdiv[2][p], R(1.0),
      [&](int kk, int d) {
        const int q = c.at(kk);
        return (a.P[1 + d][q] + a.dvh.f[d][q]) * a.ethtot0[q];
      },
      [&](int kk) {
        const int q = c.at(kk), qm = c.at(kk - 1);
        return (a.P[4][q] + rws1[q]) * (CC.afact[kk] * a.ethtot0[q] + CC.bfact[kk] * a.ethtot0[qm]);
      });
  a.dwe[2][p] = PSk(5, k) + (a.gT0e[p] + drhogetot) * R(a.dt) + (kin10 - kin11) + (PSk(0, k) - rs1[p]) * m.PHI[p];
}

template <class R>
__global__ void k_vimain_b(VimainArgs<R> a, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  if (!pole) vimain_column<R, false>(a, col_reg(i, j, l));
  else vimain_column<R, true>(a, col_pl(g, lp));
}

// ---------------------------------------------------------------------------
// elementwise helpers of the small step
// ---------------------------------------------------------------------------
// PROG_split = 0 (first stage) or PROG0 - PROG; PROG_mean = PROG[0:5]
template <class R>
__global__ void k_split_init(const R* P0a, const R* P0b, const R* P0c, const R* P0d,
                             const R* P0e, const R* P0f, Prog<R> P, R* PS0, R* PS1, R* PS2,
                             R* PS3, R* PS4, R* PS5, R* PM0, R* PM1, R* PM2,
                             R* PM3, R* PM4, int n, int first) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  const R* P0[6] = {P0a, P0b, P0c, P0d, P0e, P0f};
  R* PS[6] = {PS0, PS1, PS2, PS3, PS4, PS5};
  R* PM[5] = {PM0, PM1, PM2, PM3, PM4};
  for (int v = 0; v < 6; ++v) PS[v][t] = first ? R(0.0) : (P0[v][t] - P.v[v][t]);
  for (int v = 0; v < 5; ++v) PM[v][t] = P.v[v][t];
}

// PROG += PROG_split, then horizontalize the momentum (mod_vi.py:1572-1583)
template <class R>
__global__ void k_post(Prog<R> P, const R* PS0, const R* PS1, const R* PS2, const R* PS3,
                       const R* PS4, const R* PS5, int pole) {
  int t = (int)blockIdx.x * blockDim.x + threadIdx.x;
  const R* PS[6] = {PS0, PS1, PS2, PS3, PS4, PS5};
  int i, j, l, g, lp;
  if (!map_col(pole, t, i, j, l, g, lp)) return;
  const Col c = pole ? col_pl(g, lp) : col_reg(i, j, l);
  const bool in = !pole && interior(i, j);
  for (int k = 0; k < cD.KA; ++k) {
    int p = c.at(k);
    R v[6];
    for (int n = 0; n < 6; ++n) v[n] = P.v[n][p] + PS[n][p];
    if (pole) horiz_pl(g, lp, v[1], v[2], v[3]);
    else if (in) horiz_reg(i, j, l, v[1], v[2], v[3]);
    for (int n = 0; n < 6; ++n) P.v[n][p] = v[n];
  }
}

}  // namespace nc
