// Spring-dynamics smoothing of the icosahedral grid on the device.
//
// Restates the relaxation of prep/hgrid/mod_mkgrd.py:204-320 (MKGRD_spring):
// every interior point is pulled along the great circles to its six
// neighbours by springs of natural length dbar = beta*lambda, integrated with
// a damped explicit step, kept on the unit sphere, pentagon corners fixed,
// halos exchanged after every iteration, until max |F| / lambda < criterion.
// One iteration = one force/update kernel (double-buffered positions, block
// max of |F|/lambda folded into a device word), one halo gather and one check
// kernel; iterations are replayed from a CUDA graph in chunks and stop at the
// same iteration the host loop would (a device flag turns the remaining
// iterations of a chunk into no-ops).
#pragma once

namespace nc {

struct SpringDev {
  double *R[2][3];          // position planes (L, G, G) x/y/z, double buffered
  double *W[3];             // velocity planes (interior used)
  double *Rpl[3];           // pole points (6 * 2): index g*2 + lp
  const long long *r_dst, *r_src, *p_dst, *p_src;
  int nr, np;
  const unsigned char* sgp; // pentagon flag per region
  unsigned long long* fmax; // running max of |F|/lambda (bit pattern of a non-negative double)
  int* done;
  long long* iters;
  int G, L;
  double lam, dbar, dt, crit;
};

__device__ inline double sp_dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ inline void sp_cross(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
__device__ inline double sp_abs(const double* a) { return sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]); }

__global__ void k_spring_step(SpringDev s, int src) {
  if (*s.done) return;
  const int G = s.G, n = G - 2;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double fs = 0.0;
  if (t < (long long)s.L * n * n) {
    const int l = (int)(t / ((long long)n * n));
    const int r = (int)(t % ((long long)n * n));
    const int i = 1 + r / n, j = 1 + r % n;
    const double* const* Rin = s.R[src];
    double* const* Rout = s.R[1 - src];
    const long long plane = (long long)G * G;
    auto at = [&](int ii, int jj) { return (long long)l * plane + (long long)ii * G + jj; };
    const long long c = at(i, j);
    const double P0[3] = {Rin[0][c], Rin[1][c], Rin[2][c]};
    const bool corner = s.sgp[l] && i == 1 && j == 1;
    const int di[6] = {1, 1, 0, -1, -1, 0}, dj[6] = {0, 1, 1, 0, -1, -1};
    double Fsum[3] = {0.0, 0.0, 0.0};
    for (int m = 0; m < 6; ++m) {
      long long q = at(i + di[m], j + dj[m]);
      if (corner && m == 5) q = at(2, 1);
      const double Pm[3] = {Rin[0][q], Rin[1][q], Rin[2][q]};
      double a[3], b[3];
      sp_cross(P0, Pm, a);
      sp_cross(a, P0, b);
      const double len = sp_abs(b);
      const double dist = atan2(sp_abs(a), sp_dot(P0, Pm));
      double F[3];
      for (int d = 0; d < 3; ++d) F[d] = (dist - s.dbar) * b[d] / len;
      if (corner && m == 5) F[0] = F[1] = F[2] = 0.0;
      for (int d = 0; d < 3; ++d) Fsum[d] = (m == 0) ? F[d] : Fsum[d] + F[d];
    }
    double Wv[3] = {s.W[0][c], s.W[1][c], s.W[2][c]};
    double R0[3], W0[3];
    for (int d = 0; d < 3; ++d) R0[d] = P0[d] + Wv[d] * s.dt;
    const double rl = sp_abs(R0);
    for (int d = 0; d < 3; ++d) R0[d] = R0[d] / rl;
    for (int d = 0; d < 3; ++d) W0[d] = Wv[d] + (Fsum[d] - Wv[d]) * s.dt;
    const double E = sp_dot(R0, W0);
    for (int d = 0; d < 3; ++d) W0[d] = W0[d] - E * R0[d];
    fs = sp_abs(Fsum) / s.lam;
    if (corner) {
      for (int d = 0; d < 3; ++d) { R0[d] = P0[d]; W0[d] = 0.0; }
      fs = 0.0;
    }
    for (int d = 0; d < 3; ++d) { Rout[d][c] = R0[d]; s.W[d][c] = W0[d]; }
  }
  // block max of a non-negative double via its ordered bit pattern
  __shared__ double red[256];
  red[threadIdx.x] = fs;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + w]);
    __syncthreads();
  }
  if (threadIdx.x == 0) atomicMax(s.fmax, (unsigned long long)__double_as_longlong(red[0]));
}

// halo gather of the freshly written positions (composed plan: sources are
// never destinations, so one pass is race free)
__global__ void k_spring_comm(SpringDev s, int dstbuf) {
  if (*s.done) return;
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int G = s.G;
  double* const* R = s.R[dstbuf];
  if (t < s.nr) {
    const long long dst = s.r_dst[t], src = s.r_src[t];
    const long long di = dst % G, dj = (dst / G) % G, dl = dst / ((long long)G * G);
    const long long o = dl * G * G + di * G + dj;
    if (src >= 0) {
      const long long si = src % G, sj = (src / G) % G, sl = src / ((long long)G * G);
      const long long q = sl * G * G + si * G + sj;
      for (int d = 0; d < 3; ++d) R[d][o] = R[d][q];
    } else {
      const long long p = -src - 1;   // g*2 + lp
      for (int d = 0; d < 3; ++d) R[d][o] = s.Rpl[d][p];
    }
  } else if (t < (long long)s.nr + s.np) {
    const long long u = t - s.nr;
    const long long p = s.p_dst[u], src = s.p_src[u];
    const long long si = src % G, sj = (src / G) % G, sl = src / ((long long)G * G);
    const long long q = sl * G * G + si * G + sj;
    for (int d = 0; d < 3; ++d) s.Rpl[d][p] = R[d][q];
  }
}

__global__ void k_spring_check(SpringDev s) {
  if (*s.done) return;
  *s.iters += 1;
  const double m = __longlong_as_double((long long)*s.fmax);
  if (m < s.crit) *s.done = 1;
  *s.fmax = 0ull;
}

}  // namespace nc
