// C ABI, device memory, halo exchange and the orchestration of one NICAM-DC
// large step (RK3 HEVI, pynicamdc/nhm/dynamics/mod_dynamics.py:1725-2741).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/nicam_cuda.h"
#include "../../include/nicam_cuda_debug.h"

#include "nc_forcing.cuh"
#include "nc_tracer.cuh"
#include "nc_grid.cuh"
#include "nc_history.cuh"
#include "nc_adjoint.cuh"

using namespace nc;

static thread_local std::string g_err;
// RN(1/b) and the tail RN(1/b - RN(1/b)) for div_by: the residual 1 - b*RN(1/b)
// is exactly representable, so one fused multiply-add gives it exactly and a
// division of it by b rounds the tail correctly.
static void recip_pair(double b, double& h, double& l) {
  h = 1.0 / b;
  l = std::fma(-h, b, 1.0) / b;
}

__global__ void k_divide_known(const double* x, const double* y, double* q, int n, double b, double bh, double bl) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= n) return;
  q[t] = y ? nc::div_by(x[t], nc::recip_of(y[t])) : nc::div_by(x[t], b, bh, bl);
}

static int fail(int code, const std::string& msg) {
  g_err = msg;
  return code;
}
#define CU(call)                                                                                       \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if (e_ != cudaSuccess) return fail(NC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

#define NC_MAXCOMM 8
#define NC_KNAME 48

// ---------------------------------------------------------------------------
// halo exchange: one gather from interior / pole sources into every halo cell
// and the pole neighbour points (share/mod_comm.py:1563-1644 with the r2r,
// p2r, r2p and singular lists composed on the host, so the copy is a single
// race-free pass: no source is also a destination).
// ---------------------------------------------------------------------------
template <class R>
struct CommFields {
  R* r[NC_MAXCOMM];
  R* p[NC_MAXCOMM];
  int n;
};

template <class R>
__global__ void k_comm(CommFields<R> f, const long long* r_dst, const long long* r_src, int nr, const long long* p_dst,
                       const long long* p_src, int np) {
  // consecutive threads take consecutive entries of one level: the entries are
  // sorted by destination, so a region's halo rows are read and written in
  // contiguous runs
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int nent = nr + np;
  long long ne = (long long)nent * cD.KA;
  if (t >= ne) return;
  int k = (int)(t / nent);
  int e = (int)(t % nent);
  const long long pl = cD.plane;
  if (e < nr) {
    long long d = r_dst[e];
    long long di = ((d / pl) * cD.KA + k) * pl + d % pl;
    long long s = r_src[e];
    if (s >= 0) {
      long long si = ((s / pl) * cD.KA + k) * pl + s % pl;
      for (int n = 0; n < f.n; ++n) f.r[n][di] = f.r[n][si];
    } else {
      long long gp = -s - 1;   // g*LP + lp
      int g = (int)(gp / cD.LP), lp = (int)(gp % cD.LP);
      int pi = ipl(g, k, lp);
      for (int n = 0; n < f.n; ++n) f.r[n][di] = f.p[n][pi];
    }
  } else {
    e -= nr;
    long long gp = p_dst[e];
    int g = (int)(gp / cD.LP), lp = (int)(gp % cD.LP);
    int pi = ipl(g, k, lp);
    long long s = p_src[e];
    long long si = ((s / pl) * cD.KA + k) * pl + s % pl;
    for (int n = 0; n < f.n; ++n) f.p[n][pi] = f.r[n][si];
  }
}

// ---------------------------------------------------------------------------
// marshal kernels: host layout (i,j,k,l,v) <-> per-variable [l][k][j][i]
// ---------------------------------------------------------------------------
template <class R>
struct VarPtrs {
  R* v[NC_MAXNQ + 6];
};

// Tiled layout conversion of the regional state between the reference layout
// (i, j, k, l, v) and the device fields [v][l][k][j][i].  For one (j, k), the
// reference layout holds for every i a contiguous run over (l, v); the device
// layout holds for every (v, l) a contiguous run over i.  A block moves an
// UI x UC tile (UI values of i, UC consecutive (l, v) pairs) through shared
// memory so that both sides are read and written in contiguous runs.
#define UI 32
#define UC 128
template <class R>
__global__ void __launch_bounds__(256) k_unpack_t(const double* st, VarPtrs<R> reg, int nv) {
  __shared__ double tile[UI][UC + 1];
  const int G = cD.G, KA = cD.KA, L = cD.L;
  const int i0 = (int)blockIdx.x * UI, c0 = (int)blockIdx.y * UC;
  const int jk = (int)blockIdx.z, k = jk % KA, j = jk / KA;
  const int ncl = L * nv;
  for (int t = threadIdx.x; t < UI * UC; t += blockDim.x) {
    const int ii = t / UC, cc = t % UC;
    const int i = i0 + ii, c = c0 + cc;
    if (i < G && c < ncl) tile[ii][cc] = st[(((long long)i * G + j) * KA + k) * ncl + c];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < UI * UC; t += blockDim.x) {
    const int cc = t / UI, ii = t % UI;
    const int i = i0 + ii, c = c0 + cc;
    if (i < G && c < ncl) {
      const int l = c / nv, v = c % nv;
      reg.v[v][((l * KA + k) * G + j) * G + i] = (R)tile[ii][cc];
    }
  }
}

// The pack also looks at every value it moves: the lowest variable index
// holding a non-finite value goes to *bad (atomicMin; the caller presets it to
// a value above every index), so a download reports a non-finite state
// without another pass over the fields.
__device__ __forceinline__ void note_nonfinite(int* bad, double x, int v) {
  if (!isfinite(x)) atomicMin(bad, v);
}

template <class R>
__global__ void __launch_bounds__(256) k_pack_t(double* st, VarPtrs<R> reg, int nv, int* bad) {
  __shared__ double tile[UI][UC + 1];
  const int G = cD.G, KA = cD.KA, L = cD.L;
  const int i0 = (int)blockIdx.x * UI, c0 = (int)blockIdx.y * UC;
  const int jk = (int)blockIdx.z, k = jk % KA, j = jk / KA;
  const int ncl = L * nv;
  for (int t = threadIdx.x; t < UI * UC; t += blockDim.x) {
    const int cc = t / UI, ii = t % UI;
    const int i = i0 + ii, c = c0 + cc;
    if (i < G && c < ncl) {
      const int l = c / nv, v = c % nv;
      const double x = (double)reg.v[v][((l * KA + k) * G + j) * G + i];
      note_nonfinite(bad, x, v);
      tile[ii][cc] = x;
    }
  }
  __syncthreads();
  for (int t = threadIdx.x; t < UI * UC; t += blockDim.x) {
    const int ii = t / UC, cc = t % UC;
    const int i = i0 + ii, c = c0 + cc;
    if (i < G && c < ncl) st[(((long long)i * G + j) * KA + k) * ncl + c] = tile[ii][cc];
  }
}

// restart payloads: 64-bit byte swap between the file's big-endian stream and a field
__device__ __forceinline__ unsigned long long bswap64(unsigned long long x) {
  const unsigned lo = __byte_perm((unsigned)x, 0u, 0x0123), hi = __byte_perm((unsigned)(x >> 32), 0u, 0x0123);
  return ((unsigned long long)lo << 32) | hi;
}
__global__ void k_restart_swap(unsigned long long* dst, const unsigned long long* src, int n) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t < n) dst[t] = bswap64(src[t]);
}
// fio_read's repair of the dummy levels (nhm/share/mod_fio.py:73-84): a
// non-finite value on the top dummy level takes the level below, then one on
// the bottom dummy level takes the level above
__global__ void k_restart_dummy(double* f) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= cD.npt2i) return;
  const int G = cD.G, KA = cD.KA;
  const int i = t % G, j = (t / G) % G, l = t / (G * G);
  const int pt = ix(i, j, KA - 1, l), pb = ix(i, j, 0, l);
  if (!isfinite(f[pt])) f[pt] = f[pt - cD.planei];
  if (!isfinite(f[pb])) f[pb] = f[pb + cD.planei];
}
// COMM_var's p2r-reverse copy (share/mod_comm.py:2249-2262): the pole centre
// takes the value of the regional halo cell its designated region holds
struct PoleSrc {
  int n;
  int e[64][5];   // pole g, pole l, regional i, j, l
};
__global__ void k_pole_centre(VarPtrs<double> reg, VarPtrs<double> pol, int nv, PoleSrc ps) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  if (t >= ps.n * cD.KA) return;
  const int e = t / cD.KA, k = t % cD.KA;
  const int* r = ps.e[e];
  const int qp = ipl(r[0], k, r[1]), qr = ix(r[2], r[3], k, r[4]);
  for (int v = 0; v < nv; ++v) pol.v[v][qp] = reg.v[v][qr];
}

// the pole part of the layout conversion: (g, k, l, v) <-> fields [v][g][k][l]
template <class R>
__global__ void k_unpack_pl(const double* st_pl, VarPtrs<R> pol, int nv) {
  const int q = (int)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cD.npl) return;
  for (int v = 0; v < nv; ++v) pol.v[v][q] = (R)st_pl[(long long)q * nv + v];
}
template <class R>
__global__ void k_pack_pl(double* st_pl, VarPtrs<R> pol, int nv, int* bad) {
  const int q = (int)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= cD.npl) return;
  for (int v = 0; v < nv; ++v) {
    const double x = (double)pol.v[v][q];
    note_nonfinite(bad, x, v);
    st_pl[(long long)q * nv + v] = x;
  }
}

// finiteness of the prognostic state: the lowest variable index with a
// non-finite value (regional fields with their halo and ghost levels, then the
// pole fields) into *bad, preset to a value above every index
template <class R>
__global__ void k_finite(VarPtrs<R> reg, VarPtrs<R> pol, int nv, int* bad) {
  const int t = (int)(blockIdx.x * blockDim.x + threadIdx.x);
  const int stride = (int)(gridDim.x * blockDim.x);
  for (int v = 0; v < nv; ++v) {
    bool ok = true;
    for (int p = t; p < cD.npti; p += stride) ok = ok && isfinite(reg.v[v][p]);
    for (int p = t; p < cD.npl; p += stride) ok = ok && isfinite(pol.v[v][p]);
    if (!ok) atomicMin(bad, v);
  }
}

// ---------------------------------------------------------------------------
// global sums with Neumaier compensation (nhm/share/mod_embudget.py:74-80)
// ---------------------------------------------------------------------------
__device__ __forceinline__ void neu_add(double& s, double& c, double x) {
  double t = s + x;
  if (fabs(s) >= fabs(x)) c += (s - t) + x;
  else c += (x - t) + s;
  s = t;
}

template <class R>
__global__ void k_mass(const R* rhog, const R* rhogq, const double* vol, const R* rhog_pl,
                       const R* rhogq_pl, const double* vol_pl, double* part) {
  // part[block*2 + {0,1}] = (sum, compensation) of rho*VOLUME (rhogq given: rho*q*VOLUME)
  __shared__ double ss[256], sc[256];
  long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double s = 0.0, c = 0.0;
  int i, j, l;
  const R* num = rhogq ? rhogq : rhog;
  if (col_of(t, i, j, l)) {
    if (interior(i, j)) {
      for (int k = cD.kmin; k <= cD.kmax; ++k) {
        long long p = ix(i, j, k, l);
        neu_add(s, c, (double)num[p] / cG.GSGAM2[p] * vol[p]);
      }
    }
  } else if (t - cD.npt2 < cD.LP) {
    int lp = (int)(t - cD.npt2);
    const R* nump = rhogq_pl ? rhogq_pl : rhog_pl;
    for (int k = cD.kmin; k <= cD.kmax; ++k) {
      int p = ipl(0, k, lp);
      neu_add(s, c, (double)nump[p] / cG.GSGAM2_pl[p] * vol_pl[p]);
    }
  }
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0.0, C = 0.0;
    for (int n = 0; n < (int)blockDim.x; ++n) {
      neu_add(S, C, ss[n]);
      C += sc[n];
    }
    part[blockIdx.x * 2 + 0] = S;
    part[blockIdx.x * 2 + 1] = C;
  }
}

// ---------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------
// One field: regional and pole arrays.  The pointers hold the device
// addresses; the element type is float64, or float32 for the work fields of a
// mixed-precision handle (RG/PL give the typed view).
struct FieldPair {
  double* r = nullptr;
  double* p = nullptr;
};
template <class R>
static inline R* RG(const FieldPair& f) { return reinterpret_cast<R*>(f.r); }
template <class R>
static inline R* PL(const FieldPair& f) { return reinterpret_cast<R*>(f.p); }

// Threads per block of the column / point kernels: chosen at run time (the
// autotuner, nc_set_block), within each kernel's launch bound.
enum {
  TB_DIAG, TB_VISOLVE, TB_VIENERGY, TB_VP0C, TB_GTEND, TB_HDIFF1, TB_POST, TB_SPLIT, TB_TRC_VFLUX, TB_TRC_VADV,
  TB_TRC_REMAP, TB_TRC_QOUT, TB_TRC_APPLY, TB_TRC_RHOG, TB_N
};
static const char* const kTuneName[TB_N] = {"diag", "vi_solve", "vi_energy", "vp0_c", "gtend", "hdiff1", "post",
                                            "split_init", "trc_vflux", "trc_vadv", "trc_remap", "trc_qout",
                                            "trc_apply", "trc_rhog"};
static const int kTuneMax[TB_N] = {128, 128, 128, NC_VP0C_BLOCK, 1024, 1024, 1024, 1024, 1024, 1024, 1024, 1024,
                                   1024, 1024};

// "no non-finite value seen": every byte 0x7f, above any variable index
#define NC_BAD_NONE 0x7f7f7f7f

struct nc_handle {
  Dims D{};
  Consts C{};
  Geom Gm{};
  int blk[TB_N] = {128, 128, 128, NC_VP0C_BLOCK, 128, 128, 128, 128, 128, 128, 128, 128, 128, 128};
  // mixed precision: float32 work fields, geometry and constants (the
  // deviations pregd/rhogd and the implicit matrix Mc/Mu/Ml stay float64)
  bool mixed = false;
  ConstsT<float> Cf{};
  GeomT<float> Gmf{};
  std::map<std::string, int> field_esize;   // bytes per element of each named field
  std::vector<void*> allocs;          // everything cudaMalloc'd
  std::map<std::string, FieldPair> fields;
  cudaStream_t stream = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  bool use_graph = true;
  bool have_state = false;
  int sstep[4] = {0, 0, 0, 0};
  int nstage = 0;
  double dtl = 0, dts = 0;
  // halo plan
  long long *r_dst = nullptr, *r_src = nullptr, *p_dst = nullptr, *p_src = nullptr;
  int nr = 0, np = 0;
  // marshal staging
  double *stage = nullptr, *stage_pl = nullptr;
  double* mass_part = nullptr;
  int mass_blocks = 0;
  // non-finite detection: device slot (lowest variable index seen, NC_BAD_NONE
  // if none) and its pinned host copy, written by the downloads' pack kernels
  int* bad = nullptr;
  int* bad_host = nullptr;
  double* vol = nullptr;
  double* vol_pl = nullptr;
  long long launches = 0;
  long long graph_kernels = 0;
  int stop_phase = 0;   // debugging: end run_step after this many phases (0 = full step)
  int phase = 0;
  // state + work fields
  FieldPair P[6], Pq[NC_MAXNQ], P0[6];
  FieldPair pre, tem, vx, vy, vz, w, rho, ein, eth, pregd, rhogd, vv[3];
  FieldPair gadv[4], vt[6], vt2[6], gT0[6], frhog;
  FieldPair PSa[6], PSb[6], PM[5], vtmp2[3], gT[6], Mc, Mu, Ml, ethtot0, hdiv[3];
  FieldPair flx_v, rhog_t, flx[6], xc[9], ch[6], cm[6], q, gq[3], qa[3], Qmin, Qmax;
  FieldPair vph[8];             // horizontal terms of vp0 (div1, div2, dd, dpg)
  const double* hs_lat = nullptr;   // Held-Suarez latitude planes (optional)
  // DCMIP forcing with Kessler microphysics (optional): full-level heights,
  // the precipitation rate of the last forcing step, the forcing's flags
  const double* kess_zf = nullptr;
  double* kess_precip = nullptr;
  int kess_negative_fixer = 0, kess_update_tot_dens = 1;
  int kess_n_cl = -1, kess_n_cl2 = -1;      // terminator toy chemistry tracers (optional)
  const double *kess_lat = nullptr, *kess_lon = nullptr;
  int kess_on = 1, sm_on = 0, sm_lsc = 0;   // DCMIP schemes: Kessler, simple physics, its condensation
  int sm_bryan = 0;                         // the simple physics with the Bryan boundary layer
  int dcmip_hs = 0;                         // moist Held-Suarez on top of the DCMIP schemes
  const double* dcmip_hs_lat = nullptr;
  const double *sm_zh = nullptr, *sm_zsfc = nullptr, *sm_tsurf = nullptr, *sm_ij = nullptr;
  // derived history diagnostics (optional setup; nc_history_vars)
  bool hist = false;
  const double *hist_hgt = nullptr, *hist_coslat = nullptr, *hist_zsfc = nullptr, *hist_area = nullptr;
  const double *hist_IJ = nullptr, *hist_dgz = nullptr;
  double hist_c[10] = {};
  int hist_trc[6] = {-1, -1, -1, -1, -1, -1};   // I_QV, I_QC, I_QR, I_QI, I_QS, I_QG
  int hist_chem[2] = {-1, -1};                   // NCHEM_STR, NCHEM_END (the chemistry's columns)
  double* hist_out[H_N] = {};                    // device outputs, allocated on first request
  double* hist_old[5] = {};                      // previous outputs of the tendency fields
  bool hist_old_set[5] = {};
  double* hist_thmean = nullptr;
  bool hist_has_nstep = false;
  long long hist_nstep = 0;
  // offline tracer advection (integ_type TRCADV, DCMIP2012 test 1-1 winds)
  bool trcadv = false;
  bool trcadv_hadley = false;   // the DCMIP 1-2 winds instead of 1-1
  double* trc_time = nullptr;       // model time of the prescribed winds (device scalar)
  const double *trc_lon = nullptr, *trc_lat = nullptr, *trc_zf = nullptr, *trc_zh = nullptr;
  const double *trc_lon_pl = nullptr, *trc_lat_pl = nullptr, *trc_zf_pl = nullptr, *trc_zh_pl = nullptr;
  // the pole columns run on a second stream between the operations that mix
  // regional and pole data (halo exchanges, tracer density update)
  cudaStream_t stream2 = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // host<->device copies on their own streams (one per direction), so that a
  // state upload or download overlaps the steps on the library stream; the
  // download stages through its own buffer
  cudaStream_t s_h2d = nullptr, s_d2h = nullptr;
  cudaEvent_t ev_in_ready = nullptr, ev_in_free = nullptr, ev_out_ready = nullptr, ev_out_done = nullptr;
  cudaEvent_t ev_user = nullptr;   // ordering against a caller's stream (device-pointer marshal)
  double *stage_out = nullptr, *stage_out_pl = nullptr;
  double* adj_work = nullptr;   // exchanged copy of the Laplacian's input (allocated on first use)
  double* adj_work6 = nullptr;   // the diffusion / divergence-damping adjoints' triangle cotangents (6 fields)
  double* adj_work4 = nullptr;   // exchanged copy of the 3-D divergence damping's four momenta (first use)
  double* adj_work3 = nullptr;  // exchanged copy of the divergence's three components (first use)
  // linearised tracer step (nc_trc_step_lin): work fields allocated on first use
  FieldPair lin[20];
  bool lin_ready = false;
  bool stepped = false;   // a step has run: PM, P0 and frhog hold its winds and densities
  bool single = false;    // pole kernels on the library stream (no second stream)
  // per-kernel timing (opt-in, eager launches only): an event after every
  // launch; a kernel's time is the gap to the previous event on the stream
  bool prof = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<const char*> ev_name;
  size_t ev_used = 0;
  std::map<std::string, std::pair<double, long long>> kstats;
};

static nc_handle* g_current = nullptr;   // handle whose constants are loaded

static int dev_alloc_bytes(nc_handle* h, void** p, size_t bytes) {
  CU(cudaMalloc(p, bytes));
  h->allocs.push_back(*p);
  CU(cudaMemset(*p, 0, bytes));
  return 0;
}
static int dev_alloc(nc_handle* h, double** p, size_t n) {
  return dev_alloc_bytes(h, (void**)p, n * sizeof(double));
}

// a named field of npt regional and npl pole values: float32 in a mixed
// handle unless f64 is set, else float64
static int field(nc_handle* h, FieldPair& f, const char* name, bool f64 = false) {
  const size_t es = (h->mixed && !f64) ? sizeof(float) : sizeof(double);
  int rc = dev_alloc_bytes(h, (void**)&f.r, (size_t)h->D.npt * es);
  if (rc) return rc;
  rc = dev_alloc_bytes(h, (void**)&f.p, (size_t)h->D.npl * es);
  if (rc) return rc;
  h->fields[name] = f;
  h->field_esize[name] = (int)es;
  return 0;
}

// ---- setup array lookup / layout conversion -------------------------------
struct ArrTab {
  std::map<std::string, const nc_array*> m;
  const nc_array* get(const char* n) const {
    auto it = m.find(n);
    return it == m.end() ? nullptr : it->second;
  }
};

static int64_t numel(const nc_array* a) {
  int64_t n = 1;
  for (int d = 0; d < a->ndim; ++d) n *= a->shape[d];
  return n;
}

static int scalar(const ArrTab& T, const char* name, double& out) {
  const nc_array* a = T.get(name);
  if (!a || numel(a) < 1) return fail(NC_ERR_ARG, std::string("missing scalar ") + name);
  if (a->dtype == NC_F64) out = ((const double*)a->data)[0];
  else if (a->dtype == NC_I32) out = ((const int32_t*)a->data)[0];
  else if (a->dtype == NC_I64) out = (double)((const int64_t*)a->data)[0];
  else out = ((const uint8_t*)a->data)[0];
  return 0;
}

// regional array (i, j, kk, l, trailing...) -> device [c][l][kk][j][i]
static int up_reg(nc_handle* h, const ArrTab& T, const char* name, int kk, int ncomp, const double** out) {
  const nc_array* a = T.get(name);
  const Dims& D = h->D;
  if (!a || a->dtype != NC_F64) return fail(NC_ERR_ARG, std::string("missing float64 array ") + name);
  if (a->ndim < 4 || a->shape[0] != D.G || a->shape[1] != D.G || a->shape[2] != kk || a->shape[3] != D.L ||
      numel(a) != (int64_t)D.G * D.G * kk * D.L * ncomp)
    return fail(NC_ERR_ARG, std::string("bad shape of ") + name);
  const double* src = (const double*)a->data;
  size_t n = (size_t)numel(a);
  std::vector<double> tmp(n);
  for (int i = 0; i < D.G; ++i)
    for (int j = 0; j < D.G; ++j)
      for (int k = 0; k < kk; ++k)
        for (int l = 0; l < D.L; ++l)
          for (int c = 0; c < ncomp; ++c) {
            size_t s = ((((size_t)i * D.G + j) * kk + k) * D.L + l) * ncomp + c;
            size_t d = ((((size_t)c * D.L + l) * kk + k) * D.G + j) * D.G + i;
            tmp[d] = src[s];
          }
  double* dp;
  int rc = dev_alloc(h, &dp, n);
  if (rc) return rc;
  CU(cudaMemcpy(dp, tmp.data(), n * sizeof(double), cudaMemcpyHostToDevice));
  *out = dp;
  return 0;
}

// pole array uploaded in its own (reference) layout
static int up_pl(nc_handle* h, const ArrTab& T, const char* name, int64_t expect, const double** out) {
  const nc_array* a = T.get(name);
  if (!a || a->dtype != NC_F64) return fail(NC_ERR_ARG, std::string("missing float64 array ") + name);
  if (numel(a) != expect) return fail(NC_ERR_ARG, std::string("bad size of ") + name);
  double* dp;
  int rc = dev_alloc(h, &dp, (size_t)expect);
  if (rc) return rc;
  CU(cudaMemcpy(dp, a->data, (size_t)expect * sizeof(double), cudaMemcpyHostToDevice));
  *out = dp;
  return 0;
}

static int up_vec(const ArrTab& T, const char* name, int n, double* dst) {
  const nc_array* a = T.get(name);
  if (!a || a->dtype != NC_F64 || numel(a) != n) return fail(NC_ERR_ARG, std::string("bad 1-d array ") + name);
  std::memcpy(dst, a->data, n * sizeof(double));
  return 0;
}

// The run constants and geometry pointers are device-global (__constant__), so
// a handle's kernels read whatever handle is current when they run.  Before
// another handle's tables are loaded, the previously current handle's queued
// work (steps, marshal kernels, copies) must have finished: its streams are
// non-blocking, so nothing else orders them before the constant copy.
static int drain(nc_handle* h) {
  for (cudaStream_t st : {h->stream, h->stream2, h->s_h2d, h->s_d2h})
    if (st) CU(cudaStreamSynchronize(st));
  return 0;
}

static int load_consts(nc_handle* h) {
  if (g_current == h) return 0;
  if (g_current) {
    int rc = drain(g_current);
    if (rc) return rc;
  }
  CU(cudaMemcpyToSymbol(cD, &h->D, sizeof(Dims)));
  CU(cudaMemcpyToSymbol(cC, &h->C, sizeof(Consts)));
  CU(cudaMemcpyToSymbol(cG, &h->Gm, sizeof(Geom)));
  if (h->mixed) {
    CU(cudaMemcpyToSymbol(cCf, &h->Cf, sizeof(ConstsT<float>)));
    CU(cudaMemcpyToSymbol(cGf, &h->Gmf, sizeof(GeomT<float>)));
  }
  g_current = h;
  return 0;
}

#define TRY(x)            \
  do {                    \
    int rc_ = (x);        \
    if (rc_) return rc_;  \
  } while (0)

// ---------------------------------------------------------------------------
// launch helpers
// ---------------------------------------------------------------------------
static const int kBlock = 128;
static unsigned grid_cols_kl(const nc_handle* h) {   // regional columns + (k, lp) pole threads
  long long n = h->D.npt2 + (long long)h->D.KA * h->D.LP;
  return (unsigned)((n + kBlock - 1) / kBlock);
}

static int mark(nc_handle* h, const char* what) {
  if (h->ev_used == h->ev_pool.size()) {
    cudaEvent_t e;
    CU(cudaEventCreate(&e));
    h->ev_pool.push_back(e);
    h->ev_name.push_back(nullptr);
  }
  CU(cudaEventRecord(h->ev_pool[h->ev_used], h->stream));
  h->ev_name[h->ev_used] = what;
  h->ev_used++;
  return 0;
}

static int check_launch(nc_handle* h, const char* what) {
  h->launches++;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(NC_ERR_CUDA, std::string("launch ") + what + ": " + cudaGetErrorString(e));
  if (h->prof) return mark(h, what);
  return 0;
}

// fold the events of one profiled step into the per-kernel totals
static int collect_profile(nc_handle* h) {
  CU(cudaStreamSynchronize(h->stream));
  for (size_t n = 1; n < h->ev_used; ++n) {
    if (!h->ev_name[n]) continue;
    float ms = 0.f;
    CU(cudaEventElapsedTime(&ms, h->ev_pool[n - 1], h->ev_pool[n]));
    auto& st = h->kstats[h->ev_name[n]];
    st.first += ms;
    st.second += 1;
  }
  h->ev_used = 0;
  return 0;
}

#define TRY_(x)           \
  do {                    \
    int rc_ = (x);        \
    if (rc_) return rc_;  \
  } while (0)

static int fork_pl(nc_handle* h) {
  if (h->prof || h->single || !h->stream2) return 0;
  CU(cudaEventRecord(h->ev_fork, h->stream));
  CU(cudaStreamWaitEvent(h->stream2, h->ev_fork, 0));
  return 0;
}
static int join_pl(nc_handle* h) {
  if (h->prof || h->single || !h->stream2) return 0;
  CU(cudaEventRecord(h->ev_join, h->stream2));
  CU(cudaStreamWaitEvent(h->stream, h->ev_join, 0));
  return 0;
}
static cudaStream_t pole_stream(nc_handle* h) {
  return (h->prof || h->single || !h->stream2) ? h->stream : h->stream2;
}

template <class R>
static int comm(nc_handle* h, std::initializer_list<FieldPair> fl) {
  CommFields<R> f{};
  f.n = 0;
  for (const FieldPair& p : fl) {
    f.r[f.n] = RG<R>(p);
    f.p[f.n] = PL<R>(p);
    f.n++;
  }
  long long ne = (long long)(h->nr + h->np) * h->D.KA;
  unsigned g = (unsigned)((ne + 255) / 256);
  TRY_(join_pl(h));
  k_comm<<<g, 256, 0, h->stream>>>(f, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
  TRY_(check_launch(h, "comm"));
  return fork_pl(h);
}

template <class R>
static Prog<R> prog_reg(nc_handle* h) {
  Prog<R> p;
  for (int v = 0; v < 6; ++v) p.v[v] = RG<R>(h->P[v]);
  return p;
}
template <class R>
static Prog<R> prog_pl(nc_handle* h) {
  Prog<R> p;
  for (int v = 0; v < 6; ++v) p.v[v] = PL<R>(h->P[v]);
  return p;
}

// ---------------------------------------------------------------------------
// one large step (mod_dynamics.py:1725-2741, numpy path)
// ---------------------------------------------------------------------------
#define PHASE()                                                                   \
  do {                                                                            \
    if (h->stop_phase > 0 && ++h->phase >= h->stop_phase) return join_pl(h);      \
  } while (0)

// halo exchange of the whole PRG_var: PROG and every tracer
template <class R>
static int comm_prg(nc_handle* h) {
  const Dims& D = h->D;
  CommFields<R> f{};
  int n = 0;
  for (int v = 0; v < 6; ++v) { f.r[n] = RG<R>(h->P[v]); f.p[n] = PL<R>(h->P[v]); n++; }
  for (int iq = 0; iq < D.nq && n < NC_MAXCOMM; ++iq) { f.r[n] = RG<R>(h->Pq[iq]); f.p[n] = PL<R>(h->Pq[iq]); n++; }
  f.n = n;
  long long ne = (long long)(h->nr + h->np) * D.KA;
  TRY(join_pl(h));
  k_comm<<<(unsigned)((ne + 255) / 256), 256, 0, h->stream>>>(f, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
  TRY(check_launch(h, "comm_final"));
  for (int iq = NC_MAXCOMM - 6; iq < D.nq; ++iq) TRY(comm<R>(h, {h->Pq[iq]}));
  return 0;
}

// ---------------------------------------------------------------------------
// the tracer advection of a step (mod_src_tracer.py:83-1228) in its parts:
// vertical mass fluxes and the density after the vertical half step, the
// vertical advection of one tracer, the horizontal fluxes, Courant numbers and
// face centroids, the horizontal advection with the Thuburn limiter of one
// tracer, and the density after the horizontal step.  The winds are PM, the
// density at the step's start P0[0], the density tendency frhog.
// ---------------------------------------------------------------------------
template <class R>
static int trc_vflux(nc_handle* h) {
  const Dims& D = h->D;
  const cudaStream_t s = h->stream, ps = pole_stream(h);
  const unsigned pcb = (unsigned)((6 * D.LP + 31) / 32);
  const double dt = h->dtl;
  for (int pole = 0; pole < 2; ++pole) {
    TrcFluxArgs<R> ta;
    auto F = [&](FieldPair& f) { return pole ? PL<R>(f) : RG<R>(f); };
    ta.rvx = F(h->PM[1]); ta.rvy = F(h->PM[2]); ta.rvz = F(h->PM[3]); ta.rw = F(h->PM[4]);
    ta.rhog_in = F(h->P0[0]); ta.frhog = F(h->frhog); ta.flx_v = F(h->flx_v); ta.rhog_t = F(h->rhog_t);
    ta.dt = dt;
    if (!pole) k_trc_vflux<<<(unsigned)((D.npt2 + h->blk[TB_TRC_VFLUX] - 1) / h->blk[TB_TRC_VFLUX]), h->blk[TB_TRC_VFLUX], 0, s>>>(ta, 0);
    else k_trc_vflux<<<pcb, 32, 0, ps>>>(ta, 1);
    TRY(check_launch(h, pole ? "trc_vflux_pl" : "trc_vflux"));
  }
  return 0;
}

// vertical advection of the tracer mass x in place: the first (second) step
// of the tracer advection, density P0[0] (rhog_t), no clamp (clamp)
template <class R>
static int trc_vadv(nc_handle* h, FieldPair& x, bool second) {
  const Dims& D = h->D;
  const cudaStream_t s = h->stream, ps = pole_stream(h);
  const unsigned pcb = (unsigned)((6 * D.LP + 31) / 32);
  const double dt = h->dtl;
  for (int pole = 0; pole < 2; ++pole) {
    TrcVadvArgs<R> va;
    auto F = [&](FieldPair& f) { return pole ? PL<R>(f) : RG<R>(f); };
    va.rhogq = F(x);
    va.den = second ? F(h->rhog_t) : F(h->P0[0]);
    va.flx_v = F(h->flx_v); va.frhog = F(h->frhog);
    va.dt = dt; va.bcoef = 0.0; va.clamp = second ? 1 : 0; va.dtl = dt;
    if (!pole) k_trc_vadv<<<(unsigned)((D.npt2 + h->blk[TB_TRC_VADV] - 1) / h->blk[TB_TRC_VADV]), h->blk[TB_TRC_VADV], 0, s>>>(va, 0);
    else k_trc_vadv<<<pcb, 32, 0, ps>>>(va, 1);
    TRY(check_launch(h, pole ? "trc_vadv_pl" : "trc_vadv"));
  }
  return 0;
}

template <class R>
static int trc_hflux(nc_handle* h) {
  const Dims& D = h->D;
  const cudaStream_t s = h->stream, ps = pole_stream(h);
  const unsigned pkb = (unsigned)((D.KA * D.LP + 127) / 128);
  const double dt = h->dtl;
  {
    TrcHfluxArgs<R> ha;
    ha.rho = RG<R>(h->PM[0]); ha.rvx = RG<R>(h->PM[1]); ha.rvy = RG<R>(h->PM[2]); ha.rvz = RG<R>(h->PM[3]); ha.rhog_t = RG<R>(h->rhog_t);
    for (int f = 0; f < 6; ++f) { ha.flx[f] = RG<R>(h->flx[f]); ha.ch[f] = RG<R>(h->ch[f]); ha.cm[f] = RG<R>(h->cm[f]); }
    for (int f = 0; f < 9; ++f) ha.xc[f] = RG<R>(h->xc[f]);
    ha.dt = dt;
    {
      const dim3 gt((unsigned)D.KA, (unsigned)(((D.G + TH_DX - 1) / TH_DX) * ((D.G + TH_DY - 1) / TH_DY)), (unsigned)D.L);
      k_trc_hflux_t<<<gt, TH_DX * TH_DY, 0, s>>>(ha);
    }
    TRY(check_launch(h, "trc_hflux"));
    TrcHfluxPlArgs<R> hp;
    hp.rho = PL<R>(h->PM[0]); hp.rvx = PL<R>(h->PM[1]); hp.rvy = PL<R>(h->PM[2]); hp.rvz = PL<R>(h->PM[3]); hp.rhog_t = PL<R>(h->rhog_t);
    hp.flx = PL<R>(h->flx[0]); hp.xc = PL<R>(h->xc[0]); hp.ch = PL<R>(h->ch[0]); hp.cm = PL<R>(h->cm[0]); hp.dt = dt;
    k_trc_hflux_pl<<<pkb, 128, 0, ps>>>(hp);
    TRY(check_launch(h, "trc_hflux_pl"));
  }
  return 0;
}

// horizontal advection of the tracer mass x in place (gradient, exchange, face
// values, Qout, exchange, flux update); leaves q, gq, qa, Qmin / Qmax behind
template <class R>
static int trc_horizontal(nc_handle* h, FieldPair& x) {
  const Dims& D = h->D;
  const cudaStream_t s = h->stream, ps = pole_stream(h);
  const unsigned pkb = (unsigned)((D.KA * D.LP + 127) / 128);
  const double dt = h->dtl;
  {
    const dim3 gt((unsigned)D.KA, (unsigned)(((D.G - 2 + TG_DX - 1) / TG_DX) * ((D.G - 2 + TG_DY - 1) / TG_DY)),
                  (unsigned)D.L);
    k_trc_grad_t<<<gt, TG_DX * TG_DY, 0, s>>>(RG<R>(x), RG<R>(h->rhog_t), RG<R>(h->q), RG<R>(h->gq[0]), RG<R>(h->gq[1]),
                                              RG<R>(h->gq[2]));
  }
  TRY(check_launch(h, "trc_grad"));
  k_trc_grad_pl<<<pkb, 128, 0, ps>>>(PL<R>(x), PL<R>(h->rhog_t), PL<R>(h->q), PL<R>(h->gq[0]), PL<R>(h->gq[1]), PL<R>(h->gq[2]));
  TRY(check_launch(h, "trc_grad_pl"));
  TRY(comm<R>(h, {h->gq[0], h->gq[1], h->gq[2]}));
  TrcRemapArgs<R> ra;
  ra.q = RG<R>(h->q); ra.gq0 = RG<R>(h->gq[0]); ra.gq1 = RG<R>(h->gq[1]); ra.gq2 = RG<R>(h->gq[2]);
  for (int f = 0; f < 9; ++f) ra.xc[f] = RG<R>(h->xc[f]);
  for (int f = 0; f < 6; ++f) ra.cm[f] = RG<R>(h->cm[f]);
  for (int f = 0; f < 3; ++f) ra.qa[f] = RG<R>(h->qa[f]);
  k_trc_remap<<<(unsigned)((D.npt2 + h->blk[TB_TRC_REMAP] - 1) / h->blk[TB_TRC_REMAP]), h->blk[TB_TRC_REMAP], 0, s>>>(ra);
  TRY(check_launch(h, "trc_remap"));
  TrcRemapPlArgs<R> rp;
  rp.q = PL<R>(h->q); rp.gq0 = PL<R>(h->gq[0]); rp.gq1 = PL<R>(h->gq[1]); rp.gq2 = PL<R>(h->gq[2]); rp.xc = PL<R>(h->xc[0]);
  rp.cm = PL<R>(h->cm[0]); rp.qa = PL<R>(h->qa[0]);
  k_trc_remap_pl<<<pkb, 128, 0, ps>>>(rp);
  TRY(check_launch(h, "trc_remap_pl"));
  TrcLimArgs<R> la;
  la.q = RG<R>(h->q); la.rhog_t = RG<R>(h->rhog_t); la.frhog = RG<R>(h->frhog);
  for (int f = 0; f < 6; ++f) { la.ch[f] = RG<R>(h->ch[f]); la.cm[f] = RG<R>(h->cm[f]); la.flx[f] = RG<R>(h->flx[f]); }
  for (int f = 0; f < 3; ++f) la.qa[f] = RG<R>(h->qa[f]);
  la.qout_min = RG<R>(h->Qmin); la.qout_max = RG<R>(h->Qmax); la.Qmin = RG<R>(h->Qmin); la.Qmax = RG<R>(h->Qmax);
  la.rhogq = RG<R>(x); la.dt = dt;
  TrcLimPlArgs<R> lp;
  lp.q = PL<R>(h->q); lp.ch = PL<R>(h->ch[0]); lp.cm = PL<R>(h->cm[0]); lp.rhog_t = PL<R>(h->rhog_t); lp.frhog = PL<R>(h->frhog);
  lp.qa = PL<R>(h->qa[0]); lp.flx = PL<R>(h->flx[0]); lp.Qmin = PL<R>(h->Qmin); lp.Qmax = PL<R>(h->Qmax);
  lp.qout_min = PL<R>(h->Qmin); lp.qout_max = PL<R>(h->Qmax); lp.rhogq = PL<R>(x); lp.dt = dt;
  k_trc_qout<<<(unsigned)((D.npt2 + h->blk[TB_TRC_QOUT] - 1) / h->blk[TB_TRC_QOUT]), h->blk[TB_TRC_QOUT], 0, s>>>(la);
  TRY(check_launch(h, "trc_qout"));
  k_trc_qout_pl<<<pkb, 128, 0, ps>>>(lp);
  TRY(check_launch(h, "trc_qout_pl"));
  TRY(comm<R>(h, {h->Qmin, h->Qmax}));
  k_trc_apply<<<(unsigned)((D.npt2 + h->blk[TB_TRC_APPLY] - 1) / h->blk[TB_TRC_APPLY]), h->blk[TB_TRC_APPLY], 0, s>>>(la);
  TRY(check_launch(h, "trc_apply"));
  k_trc_apply_pl<<<pkb, 128, 0, ps>>>(lp);
  TRY(check_launch(h, "trc_apply_pl"));
  return 0;
}

template <class R>
static int trc_rhog(nc_handle* h) {
  const Dims& D = h->D;
  const cudaStream_t s = h->stream;
  const double dt = h->dtl;
  TRY(join_pl(h));
  k_trc_rhog<<<(unsigned)(((D.npt2 + (long long)D.KA * D.LP) + h->blk[TB_TRC_RHOG] - 1) / h->blk[TB_TRC_RHOG]), h->blk[TB_TRC_RHOG], 0, s>>>(RG<R>(h->rhog_t), RG<R>(h->flx[0]), RG<R>(h->flx[1]), RG<R>(h->flx[2]), RG<R>(h->flx[3]), RG<R>(h->flx[4]),
                                     RG<R>(h->flx[5]), RG<R>(h->frhog), (R)dt, PL<R>(h->flx[0]), PL<R>(h->rhog_t), PL<R>(h->frhog));
  TRY(check_launch(h, "trc_rhog"));
  TRY(fork_pl(h));
  return 0;
}

template <class R>
static int run_step(nc_handle* h) {
  cudaStream_t s = h->stream;
  const cudaStream_t ps = pole_stream(h);
  h->phase = 0;
  const Dims& D = h->D;
  const unsigned gkl = grid_cols_kl(h);
  // pole kernels: one thread per pole column (6 * LP) or per pole level (kall * LP);
  // LP = 2 per ensemble member
  const unsigned pcb = (unsigned)((6 * D.LP + 31) / 32);
  const unsigned pkb = (unsigned)((D.KA * D.LP + 127) / 128);
  const unsigned npt_blocks = (unsigned)((D.npt + kBlock - 1) / kBlock);
  const unsigned npl_blocks = (unsigned)((D.npl + kBlock - 1) / kBlock);
  // per-level tiled kernels: (levels kmin..kmax, tiles, regions)
  const dim3 vagrid((unsigned)((D.kmax - D.kmin + VA_NK) / VA_NK),
                    (unsigned)(((D.G - 2 + DD_DX - 1) / DD_DX) * ((D.G - 2 + DD_DY - 1) / DD_DY)), (unsigned)D.L);
  const dim3 lvgrid((unsigned)(D.kmax - D.kmin + 1),
                    (unsigned)(((D.G - 2 + DD_DX - 1) / DD_DX) * ((D.G - 2 + DD_DY - 1) / DD_DY)), (unsigned)D.L);
  const dim3 lvgrid_vp((unsigned)(D.kmax - D.kmin + 1),
                       (unsigned)(((D.G - 2 + VP_DX - 1) / VP_DX) * ((D.G - 2 + VP_DY - 1) / VP_DY)), (unsigned)D.L);
  // PROG0 = PROG at the start of the step (mod_dynamics.py:1939-1968)
  for (int v = 0; v < 6; ++v) {
    CU(cudaMemcpyAsync(RG<R>(h->P0[v]), RG<R>(h->P[v]), D.npt * sizeof(R), cudaMemcpyDeviceToDevice, s));
    CU(cudaMemcpyAsync(PL<R>(h->P0[v]), PL<R>(h->P[v]), D.npl * sizeof(R), cudaMemcpyDeviceToDevice, s));
  }
  if (h->prof) TRY(mark(h, nullptr));
  TRY(fork_pl(h));
  for (int nl = 0; nl < h->nstage; ++nl) {
    const bool last = (nl == h->nstage - 1);
    // ---- Pre_Post
    auto diag_args = [&](bool pole) {
      DiagArgs<R> a;
      a.P = pole ? prog_pl<R>(h) : prog_reg<R>(h);
      for (int n = 0; n < h->C.nqw; ++n) a.Pqw[n] = pole ? PL<R>(h->Pq[n]) : RG<R>(h->Pq[n]);
      auto F = [&](FieldPair& f) { return pole ? PL<R>(f) : RG<R>(f); };
      auto F64 = [&](FieldPair& f) { return pole ? f.p : f.r; };
      a.pre = F(h->pre); a.tem = F(h->tem); a.vx = F(h->vx); a.vy = F(h->vy); a.vz = F(h->vz); a.w = F(h->w);
      a.rho = F(h->rho); a.ein = F(h->ein); a.eth = F(h->eth); a.pregd = F64(h->pregd); a.rhogd = F64(h->rhogd);
      a.vvx = F(h->vv[0]); a.vvy = F(h->vv[1]); a.vvz = F(h->vv[2]);
      return a;
    };
    // regional and pole columns: same kernel, launched with the matching pointers
    k_diag<<<(unsigned)((D.npt2 + h->blk[TB_DIAG] - 1) / h->blk[TB_DIAG]), h->blk[TB_DIAG], 0, s>>>(diag_args(false), 0);
    TRY(check_launch(h, "diag"));
    k_diag<<<pcb, 32, 0, ps>>>(diag_args(true), 1);
    TRY(check_launch(h, "diag_pl"));
    PHASE();
    // ---- momentum advection
    AdvMomArgs<R> am;
    am.rg = RG<R>(h->P[0]); am.rvx = RG<R>(h->P[1]); am.rvy = RG<R>(h->P[2]); am.rvz = RG<R>(h->P[3]); am.rw = RG<R>(h->P[4]);
    am.vvx = RG<R>(h->vv[0]); am.vvy = RG<R>(h->vv[1]); am.vvz = RG<R>(h->vv[2]);
    am.gvx = RG<R>(h->gadv[0]); am.gvy = RG<R>(h->gadv[1]); am.gvz = RG<R>(h->gadv[2]); am.gw = RG<R>(h->gadv[3]);
    {
      // interior cells, levels kmin..kmax (see k_advmom_t)
      const dim3 gt((unsigned)(((D.G - 2 + 31) / 32) * ((D.G - 2 + 7) / 8)), 1, (unsigned)D.L);
      k_advmom_t<<<gt, 256, 0, s>>>(am);
    }
    TRY(check_launch(h, "advmom"));
    AdvMomArgs<R> amp;
    amp.rg = PL<R>(h->P[0]); amp.rvx = PL<R>(h->P[1]); amp.rvy = PL<R>(h->P[2]); amp.rvz = PL<R>(h->P[3]); amp.rw = PL<R>(h->P[4]);
    amp.vvx = PL<R>(h->vv[0]); amp.vvy = PL<R>(h->vv[1]); amp.vvz = PL<R>(h->vv[2]);
    amp.gvx = PL<R>(h->gadv[0]); amp.gvy = PL<R>(h->gadv[1]); amp.gvz = PL<R>(h->gadv[2]); amp.gw = PL<R>(h->gadv[3]);
    k_advmom_pl<<<pcb, 32, 0, ps>>>(amp);
    TRY(check_launch(h, "advmom_pl"));
    PHASE();
    // ---- hyperdiffusion
    Six<R> src, srcp;
    SixOut<R> o1, o1p;
    const FieldPair* sf[6] = {&h->vx, &h->vy, &h->vz, &h->w, &h->tem, &h->rho};
    for (int n = 0; n < 6; ++n) {
      src.f[n] = RG<R>(*sf[n]); srcp.f[n] = PL<R>(*sf[n]);
      o1.f[n] = RG<R>(h->vt[n]); o1p.f[n] = PL<R>(h->vt[n]);
    }
    k_hdiff1<<<(unsigned)((D.npt2 + h->blk[TB_HDIFF1] - 1) / h->blk[TB_HDIFF1]), h->blk[TB_HDIFF1], 0, s>>>(src, o1);
    TRY(check_launch(h, "hdiff1"));
    k_hdiff1_pl<<<pkb, 128, 0, ps>>>(srcp, o1p);
    TRY(check_launch(h, "hdiff1_pl"));
    TRY(comm<R>(h, {h->vt[0], h->vt[1], h->vt[2], h->vt[3], h->vt[4], h->vt[5]}));
    PHASE();
    Six<R> vin, vinp;
    SixOut<R> o2, o2p;
    for (int n = 0; n < 6; ++n) {
      vin.f[n] = RG<R>(h->vt[n]); vinp.f[n] = PL<R>(h->vt[n]);
      o2.f[n] = RG<R>(h->vt2[n]); o2p.f[n] = PL<R>(h->vt2[n]);
    }
    {
      // interior cells; the exchange below fills the halo rows
      const dim3 gt((unsigned)((D.G - 2 + HD_DX - 1) / HD_DX), (unsigned)((D.G - 2 + HD_DY - 1) / HD_DY),
                    (unsigned)D.L);
      const dim3 gl2((unsigned)((D.KA + HD_NK - 1) / HD_NK), gt.x * gt.y, gt.z);
      k_hdiff2_m<<<gl2, HD_DX * HD_DY, hdiff2_m_smem<R>(), s>>>(vin, RG<R>(h->P[0]), o2);
      TRY(check_launch(h, "hdiff2"));
    }
    k_hdiff2_pl<<<pkb, 128, 0, ps>>>(vinp, PL<R>(h->P[0]), o2p);
    TRY(check_launch(h, "hdiff2_pl"));
    TRY(comm<R>(h, {h->vt2[0], h->vt2[1], h->vt2[2], h->vt2[3], h->vt2[4], h->vt2[5]}));
    PHASE();
    // ---- large-step tendency
    for (int pole = 0; pole < 2; ++pole) {
      GtendArgs<R> ga;
      auto F = [&](FieldPair& f) { return pole ? PL<R>(f) : RG<R>(f); };
      for (int n = 0; n < 6; ++n) { ga.vt2.f[n] = F(h->vt2[n]); ga.gT0[n] = F(h->gT0[n]); }
      ga.lapT = F(h->vt[4]);
      ga.vx = F(h->vx); ga.vy = F(h->vy); ga.vz = F(h->vz); ga.w = F(h->w);
      ga.rhog = F(h->P[0]); ga.gvx = F(h->gadv[0]); ga.gvy = F(h->gadv[1]); ga.gvz = F(h->gadv[2]);
      ga.gw = F(h->gadv[3]); ga.frhog = F(h->frhog);
      if (!pole) k_gtend<<<(unsigned)((D.npt2 + h->blk[TB_GTEND] - 1) / h->blk[TB_GTEND]), h->blk[TB_GTEND], 0, s>>>(ga, 0);
      else k_gtend<<<pcb, 32, 0, ps>>>(ga, 1);
      TRY(check_launch(h, pole ? "gtend_pl" : "gtend"));
    }
    PHASE();
    // ---- vi_small_step (mod_vi.py:104-1590)
    k_split_init<<<(unsigned)((D.npt + h->blk[TB_SPLIT] - 1) / h->blk[TB_SPLIT]), h->blk[TB_SPLIT], 0, s>>>(RG<R>(h->P0[0]), RG<R>(h->P0[1]), RG<R>(h->P0[2]), RG<R>(h->P0[3]), RG<R>(h->P0[4]),
                                                RG<R>(h->P0[5]), prog_reg<R>(h), RG<R>(h->PSa[0]), RG<R>(h->PSa[1]), RG<R>(h->PSa[2]),
                                                RG<R>(h->PSa[3]), RG<R>(h->PSa[4]), RG<R>(h->PSa[5]), RG<R>(h->PM[0]), RG<R>(h->PM[1]),
                                                RG<R>(h->PM[2]), RG<R>(h->PM[3]), RG<R>(h->PM[4]), D.npt, nl == 0);
    TRY(check_launch(h, "split_init"));
    k_split_init<<<npl_blocks, kBlock, 0, ps>>>(PL<R>(h->P0[0]), PL<R>(h->P0[1]), PL<R>(h->P0[2]), PL<R>(h->P0[3]), PL<R>(h->P0[4]),
                                                PL<R>(h->P0[5]), prog_pl<R>(h), PL<R>(h->PSa[0]), PL<R>(h->PSa[1]), PL<R>(h->PSa[2]),
                                                PL<R>(h->PSa[3]), PL<R>(h->PSa[4]), PL<R>(h->PSa[5]), PL<R>(h->PM[0]), PL<R>(h->PM[1]),
                                                PL<R>(h->PM[2]), PL<R>(h->PM[3]), PL<R>(h->PM[4]), D.npl, nl == 0);
    TRY(check_launch(h, "split_init_pl"));
    auto dd3d = [&](FieldPair* v4) -> int {
      Four<R> v, vp;
      Three<R> o, op;
      for (int n = 0; n < 4; ++n) { v.f[n] = RG<R>(v4[n]); vp.f[n] = PL<R>(v4[n]); }
      for (int d = 0; d < 3; ++d) { o.f[d] = RG<R>(h->vtmp2[d]); op.f[d] = PL<R>(h->vtmp2[d]); }
      // interior cells only: halo rows are filled by the exchange below and the
      // boundary levels of vtmp2 stay zero from allocation
      const dim3 gt((unsigned)((D.G - 2 + DD_DX - 1) / DD_DX), (unsigned)((D.G - 2 + DD_DY - 1) / DD_DY), (unsigned)D.L);
      k_dd3d_m<R, true><<<gt, DD_DX * DD_DY, dd3d_m_smem<R>(), s>>>(v, o);
      TRY(check_launch(h, "dd3d"));
      k_dd3d_pl<<<pkb, 128, 0, ps>>>(vp, op);
      TRY(check_launch(h, "dd3d_pl"));
      return comm<R>(h, {h->vtmp2[0], h->vtmp2[1], h->vtmp2[2]});
    };
    {
      FieldPair v4[4] = {h->P[1], h->P[2], h->P[3], h->P[4]};
      TRY(dd3d(v4));
    }
    PHASE();
    for (int pole = 0; pole < 2; ++pole) {
      Vp0Args<R> va;
      auto F = [&](FieldPair& f) { return pole ? PL<R>(f) : RG<R>(f); };
      auto F64 = [&](FieldPair& f) { return pole ? f.p : f.r; };
      va.P = pole ? prog_pl<R>(h) : prog_reg<R>(h);
      va.vx = F(h->vx); va.vy = F(h->vy); va.vz = F(h->vz); va.eth = F(h->eth); va.pregd = F64(h->pregd);
      va.rhogd = F64(h->rhogd);
      for (int d = 0; d < 3; ++d) va.vt.f[d] = F(h->vtmp2[d]);
      for (int n = 0; n < 6; ++n) { va.gT0[n] = F(h->gT0[n]); va.gT[n] = F(h->gT[n]); }
      va.Mc = F64(h->Mc); va.Mu = F64(h->Mu); va.Ml = F64(h->Ml); va.ethtot0 = F(h->ethtot0);
      va.dt = h->dts;
      if (!pole) {
        Vp0H<R> vh;
        for (int n = 0; n < 8; ++n) vh.out[n] = RG<R>(h->vph[n]);
        k_vp0_hl<<<lvgrid_vp, VP_DX * VP_DY, 0, s>>>(va, vh);
        TRY(check_launch(h, "vp0_h"));
        k_vp0_cr<<<(unsigned)((D.npt2 + h->blk[TB_VP0C] - 1) / h->blk[TB_VP0C]), h->blk[TB_VP0C], 0, s>>>(va, vh);
        TRY(check_launch(h, "vp0_c"));
      } else {
        k_vp0<<<pcb, 32, 0, ps>>>(va, 1);
        TRY(check_launch(h, "vp0_pl"));
      }
    }
    PHASE();
    const int nitr = h->sstep[nl];
    const double rweight = 1.0 / (double)nitr;
    const double RovCV = h->C.Rdry / h->C.CVdry;
    for (int ns = 0; ns < nitr; ++ns) {
      FieldPair* PS = (ns % 2 == 0) ? h->PSa : h->PSb;     // current split values
      FieldPair* PN = (ns % 2 == 0) ? h->PSb : h->PSa;     // next split values
      {
        FieldPair v4[4] = {PS[1], PS[2], PS[3], PS[4]};
        TRY(dd3d(v4));
      }
      PHASE();
      for (int pole = 0; pole < 2; ++pole) {
        Path1Args<R> pa;
        auto F = [&](FieldPair& f) { return pole ? PL<R>(f) : RG<R>(f); };
        for (int n = 0; n < 6; ++n) { pa.PS[n] = F(PS[n]); pa.gT[n] = F(h->gT[n]); }
        pa.rhog = F(h->P[0]);
        for (int d = 0; d < 3; ++d) { pa.vt.f[d] = F(h->vtmp2[d]); pa.dvh[d] = F(PN[1 + d]); }
        for (int n = 0; n < 5; ++n) pa.PM[n] = F(h->PM[n]);
        pa.dt = h->dts; pa.rweight = rweight; pa.RovCV = RovCV;
        if (!pole) {
          k_path1_l<<<lvgrid, DD_DX * DD_DY, 0, s>>>(pa);
          TRY(check_launch(h, "path1"));
        } else {
          k_path1<<<pcb, 32, 0, ps>>>(pa, 1);
          TRY(check_launch(h, "path1_pl"));
        }
      }
      TRY(comm<R>(h, {PN[1], PN[2], PN[3]}));
      PHASE();
      for (int pole = 0; pole < 2; ++pole) {
        VimainArgs<R> va;
        auto F = [&](FieldPair& f) { return pole ? PL<R>(f) : RG<R>(f); };
      auto F64 = [&](FieldPair& f) { return pole ? f.p : f.r; };
        for (int n = 0; n < 6; ++n) { va.PS[n] = F(PS[n]); va.P[n] = F(h->P[n]); va.gT[n] = F(h->gT[n]); }
        va.eth = F(h->eth); va.ethtot0 = F(h->ethtot0); va.gT0e = F(h->gT0[5]);
        va.Mc = F64(h->Mc); va.Mu = F64(h->Mu); va.Ml = F64(h->Ml);
        for (int d = 0; d < 3; ++d) { va.dvh.f[d] = F(PN[1 + d]); va.hdiv[d] = F(h->hdiv[d]); }
        va.dwe[0] = F(PN[0]); va.dwe[1] = F(PN[4]); va.dwe[2] = F(PN[5]);
        va.PM0 = F(h->PM[0]); va.PM4 = F(h->PM[4]);
        va.dt = h->dts; va.rweight = rweight; va.RovCV = RovCV;
        if (!pole) {
          if constexpr (std::is_same<R, float>::value) k_vimain_a_m<<<vagrid, DD_DX * DD_DY, 0, s>>>(va);
          else k_vimain_a_l<<<lvgrid, DD_DX * DD_DY, 0, s>>>(va);
          TRY(check_launch(h, "vimain_a"));
          if (h->C.gam_unit) k_vi_solve<R, true><<<(unsigned)((D.npt2 + h->blk[TB_VISOLVE] - 1) / h->blk[TB_VISOLVE]), h->blk[TB_VISOLVE], 0, s>>>(va);
          else k_vi_solve<R, false><<<(unsigned)((D.npt2 + h->blk[TB_VISOLVE] - 1) / h->blk[TB_VISOLVE]), h->blk[TB_VISOLVE], 0, s>>>(va);
          TRY(check_launch(h, "vi_solve"));
          k_vi_energy_p<<<(unsigned)((D.npt + h->blk[TB_VIENERGY] - 1) / h->blk[TB_VIENERGY]), h->blk[TB_VIENERGY], 0, s>>>(va);
          TRY(check_launch(h, "vi_energy"));
        } else {
          k_vimain_a<<<pkb, 128, 0, ps>>>(va, 1);
          TRY(check_launch(h, "vimain_a_pl"));
          k_vimain_b<<<pcb, 32, 0, ps>>>(va, 1);
          TRY(check_launch(h, "vimain_b_pl"));
        }
      }
      TRY(comm<R>(h, {PN[0], PN[4], PN[5]}));
      PHASE();
    }
    FieldPair* PSf = (nitr % 2 == 0) ? h->PSa : h->PSb;
    k_post<<<(unsigned)((D.npt2 + h->blk[TB_POST] - 1) / h->blk[TB_POST]), h->blk[TB_POST], 0, s>>>(prog_reg<R>(h), RG<R>(PSf[0]), RG<R>(PSf[1]), RG<R>(PSf[2]), RG<R>(PSf[3]), RG<R>(PSf[4]), RG<R>(PSf[5]), 0);
    TRY(check_launch(h, "post"));
    k_post<<<pcb, 32, 0, ps>>>(prog_pl<R>(h), PL<R>(PSf[0]), PL<R>(PSf[1]), PL<R>(PSf[2]), PL<R>(PSf[3]), PL<R>(PSf[4]), PL<R>(PSf[5]), 1);
    TRY(check_launch(h, "post_pl"));
    TRY(comm<R>(h, {h->PM[0], h->PM[1], h->PM[2], h->PM[3], h->PM[4]}));
    PHASE();
    if (!last) {
      TRY(comm<R>(h, {h->P[0], h->P[1], h->P[2], h->P[3], h->P[4], h->P[5]}));
      PHASE();
      continue;
    }
  }
  if (h->trcadv) {
    // offline tracer advection (integ_type TRCADV, mod_dynamics.py:2030-2085): the
    // tracers move with the current PROG (as the mean state, rhog_in = PROG0) and
    // no density tendency
    for (int v = 0; v < 5; ++v) {
      CU(cudaMemcpyAsync(RG<R>(h->PM[v]), RG<R>(h->P[v]), D.npt * sizeof(R), cudaMemcpyDeviceToDevice, s));
      CU(cudaMemcpyAsync(PL<R>(h->PM[v]), PL<R>(h->P[v]), D.npl * sizeof(R), cudaMemcpyDeviceToDevice, s));
    }
    CU(cudaMemsetAsync(RG<R>(h->frhog), 0, D.npt * sizeof(R), s));
    CU(cudaMemsetAsync(PL<R>(h->frhog), 0, D.npl * sizeof(R), s));
    TRY(join_pl(h));
    TRY(fork_pl(h));
  }
  // ---- tracer advection (mod_src_tracer.py:83-1228), after the last RK stage
  TRY(trc_vflux<R>(h));
  // first vertical step uses the density at the start of the step; the
  // Courant numbers of the first step are those of rhog_in
  for (int iq = 0; iq < D.nq; ++iq) TRY(trc_vadv<R>(h, h->Pq[iq], false));
  PHASE();
  TRY(trc_hflux<R>(h));
  PHASE();
  for (int iq = 0; iq < D.nq; ++iq) TRY(trc_horizontal<R>(h, h->Pq[iq]));
  PHASE();
  TRY(trc_rhog<R>(h));
  for (int iq = 0; iq < D.nq; ++iq) TRY(trc_vadv<R>(h, h->Pq[iq], true));
  PHASE();
  if (h->trcadv) {
    // the prescribed winds of the next time (mod_forcing.py forcing_update)
    TRY(join_pl(h));
    k_trcadv_time<<<1, 1, 0, s>>>(h->trc_time, h->dtl);
    TRY(check_launch(h, "trcadv_time"));
    TrcWindArgs<R> w;
    for (int v = 0; v < 6; ++v) w.P.v[v] = RG<R>(h->P[v]);
    w.lon = h->trc_lon; w.lat = h->trc_lat; w.zf = h->trc_zf; w.zh = h->trc_zh; w.time = h->trc_time;
    w.a = 6371220.0; w.Rd = 287.0; w.g = 9.80616; w.pi = 3.141592653589793238;
    w.hadley = h->trcadv_hadley;
    k_trcadv_winds<<<npt_blocks, kBlock, 0, s>>>(w, 0);
    TRY(check_launch(h, "trcadv_winds"));
    for (int v = 0; v < 6; ++v) w.P.v[v] = PL<R>(h->P[v]);
    w.lon = h->trc_lon_pl; w.lat = h->trc_lat_pl; w.zf = h->trc_zf_pl; w.zh = h->trc_zh_pl;
    k_trcadv_winds<<<npl_blocks, kBlock, 0, s>>>(w, 1);
    TRY(check_launch(h, "trcadv_winds_pl"));
  }
  // marshal-out halo exchange of PRG_var (mod_dynamics.py:2726-2727)
  TRY(comm_prg<R>(h));
  TRY(join_pl(h));
  return 0;
}

// ---------------------------------------------------------------------------
// Allocation-free air/tracer mass sum (nc_mass_sum_noalloc).  Same per-block
// compensated partial sums and the same fold order as k_mass + the host fold
// of nc_mass_sums, but with all sizes passed as arguments (no handle, no
// constant memory) and the block partials kept in a file-scope device array,
// so a call allocates nothing.  Every call on a device shares this array.
// ---------------------------------------------------------------------------
#define NC_NOALLOC_MASS_MAX_BLOCKS 4096   // 4096 blocks x 256 columns = 1,048,576 columns
static __device__ __align__(256) double g_mass_scratch[NC_NOALLOC_MASS_MAX_BLOCKS * 2];

__global__ void k_mass_noalloc(const double* rhog, const double* rhogq, const double* gsgam2, const double* vol,
                               const double* rhog_pl, const double* rhogq_pl, const double* gsgam2_pl,
                               const double* vol_pl, int G, int L, int KA, int kmin, int kmax, double* part) {
  __shared__ double ss[256], sc[256];
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long ncol = (long long)L * G * G;
  double s = 0.0, c = 0.0;
  const double* num = rhogq ? rhogq : rhog;
  if (t < ncol) {
    const int i = (int)(t % G), j = (int)((t / G) % G), l = (int)(t / ((long long)G * G));
    if (i >= 1 && i <= G - 2 && j >= 1 && j <= G - 2) {
      for (int k = kmin; k <= kmax; ++k) {
        const long long p = (((long long)l * KA + k) * G + j) * G + i;
        neu_add(s, c, num[p] / gsgam2[p] * vol[p]);
      }
    }
  } else if (t - ncol < 2) {
    const int lp = (int)(t - ncol);
    const double* nump = rhogq_pl ? rhogq_pl : rhog_pl;
    for (int k = kmin; k <= kmax; ++k) {
      const int p = k * 2 + lp;   // pole point g = 0 of (g, k, lp)
      neu_add(s, c, nump[p] / gsgam2_pl[p] * vol_pl[p]);
    }
  }
  ss[threadIdx.x] = s;
  sc[threadIdx.x] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    double S = 0.0, C = 0.0;
    for (int n = 0; n < (int)blockDim.x; ++n) {
      neu_add(S, C, ss[n]);
      C += sc[n];
    }
    part[blockIdx.x * 2 + 0] = S;
    part[blockIdx.x * 2 + 1] = C;
  }
}

// one thread folds the block partials in block order (the order of the host
// fold in nc_mass_sums) and writes the sum
__global__ void k_mass_noalloc_fold(const double* part, int nblocks, double* out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  double S = 0.0, Cc = 0.0;
  for (int b = 0; b < nblocks; ++b) {
    const double x = part[b * 2];
    const double t = S + x;
    if (fabs(S) >= fabs(x)) Cc += (S - t) + x;
    else Cc += (x - t) + S;
    S = t;
    Cc += part[b * 2 + 1];
  }
  out[0] = S + Cc;
}

// device address of g_mass_scratch, looked up once per device ordinal and kept
// for the life of the process: this assumes the device's primary context is
// never reset (cudaDeviceReset) while the library is loaded, since a reset
// context would give the array a new address
static std::mutex g_scratch_mu;
static std::map<int, double*> g_scratch_addr;

static int mass_scratch_ptr(double** out) {
  int dev = -1;
  CU(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(g_scratch_mu);
  auto it = g_scratch_addr.find(dev);
  if (it != g_scratch_addr.end()) {
    *out = it->second;
    return 0;
  }
  double* ptr = nullptr;
  CU(cudaGetSymbolAddress((void**)&ptr, g_mass_scratch));
  g_scratch_addr[dev] = ptr;
  *out = ptr;
  return 0;
}

template <class R>
static VarPtrs<R> state_ptrs(nc_handle* h, bool pole) {
  VarPtrs<R> v{};
  for (int n = 0; n < 6; ++n) v.v[n] = pole ? PL<R>(h->P[n]) : RG<R>(h->P[n]);
  for (int n = 0; n < h->D.nq; ++n) v.v[6 + n] = pole ? PL<R>(h->Pq[n]) : RG<R>(h->Pq[n]);
  return v;
}

// the marshal kernels of one state (reference layout <-> fields of type R)
template <class R>
static int unpack_state(nc_handle* h, const double* st, const double* st_pl) {
  const Dims& D = h->D;
  const int nv = 6 + D.nq;
  const dim3 gt((unsigned)((D.G + UI - 1) / UI), (unsigned)((D.L * nv + UC - 1) / UC), (unsigned)(D.G * D.KA));
  k_unpack_t<<<gt, 256, 0, h->stream>>>(st, state_ptrs<R>(h, false), nv);
  TRY(check_launch(h, "unpack"));
  k_unpack_pl<<<(unsigned)((D.npl + 127) / 128), 128, 0, h->stream>>>(st_pl, state_ptrs<R>(h, true), nv);
  return check_launch(h, "unpack_pl");
}
template <class R>
static int pack_state(nc_handle* h, double* st, double* st_pl) {
  const Dims& D = h->D;
  const int nv = 6 + D.nq;
  const dim3 gt((unsigned)((D.G + UI - 1) / UI), (unsigned)((D.L * nv + UC - 1) / UC), (unsigned)(D.G * D.KA));
  k_pack_t<<<gt, 256, 0, h->stream>>>(st, state_ptrs<R>(h, false), nv, h->bad);
  TRY(check_launch(h, "pack"));
  k_pack_pl<<<(unsigned)((D.npl + 127) / 128), 128, 0, h->stream>>>(st_pl, state_ptrs<R>(h, true), nv, h->bad);
  return check_launch(h, "pack_pl");
}
template <class R>
static int finite_state(nc_handle* h) {
  k_finite<<<4 * 148, 256, 0, h->stream>>>(state_ptrs<R>(h, false), state_ptrs<R>(h, true), 6 + h->D.nq, h->bad);
  return check_launch(h, "finite");
}
template <class R>
static int mass_sum(nc_handle* h, int n) {
  const R* num = n == 0 ? nullptr : RG<R>(h->Pq[n - 1]);
  const R* nump = n == 0 ? nullptr : PL<R>(h->Pq[n - 1]);
  k_mass<<<h->mass_blocks, 256, 0, h->stream>>>(RG<R>(h->P[0]), num, h->vol, PL<R>(h->P[0]), nump, h->vol_pl,
                                                h->mass_part);
  return check_launch(h, "mass");
}
static int step_once(nc_handle* h) { return h->mixed ? run_step<float>(h) : run_step<double>(h); }
// forget the captured step (the next nc_step captures it again)
static int drop_graph(nc_handle* h) {
  if (h->gexec || h->graph) CU(cudaStreamSynchronize(h->stream));
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  h->gexec = nullptr;
  h->graph = nullptr;
  return 0;
}
// the entry points of the float64 form only
static int f64_only(nc_handle* h, const char* what) {
  if (h->mixed) return fail(NC_ERR_STATE, std::string(what) + ": not available for a mixed-precision handle");
  return 0;
}

// ---------------------------------------------------------------------------
// linearised tracer advection step (nc_trc_step_lin)
// ---------------------------------------------------------------------------
enum { LN_X0, LN_X1, LN_X2, LN_X3, LN_RHO, LN_T1, LN_T2, LN_DQ, LN_DG0, LN_DG1, LN_DG2, LN_DQA0, LN_DQA1,
       LN_DQA2, LN_DQN, LN_DQX, LN_N };
static int lin_buffers(nc_handle* h) {
  if (h->lin_ready) return 0;
  static const char* names[LN_N] = {"lin.x0", "lin.x1", "lin.x2", "lin.x3", "lin.rho", "lin.t1", "lin.t2", "lin.dq",
                                    "lin.dg0", "lin.dg1", "lin.dg2", "lin.dqa0", "lin.dqa1", "lin.dqa2",
                                    "lin.dqmin", "lin.dqmax"};
  for (int n = 0; n < LN_N; ++n) TRY(field(h, h->lin[n], names[n], true));
  h->lin_ready = true;
  return 0;
}
static int copy_in(nc_handle* h, FieldPair& dst, const double* r, const double* p) {
  CU(cudaMemcpyAsync(dst.r, r, h->D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  CU(cudaMemcpyAsync(dst.p, p, h->D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  return h->prof ? mark(h, "lin_copy") : 0;
}
static int copy_out(nc_handle* h, double* r, double* p, const FieldPair& src) {
  CU(cudaMemcpyAsync(r, src.r, h->D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  CU(cudaMemcpyAsync(p, src.p, h->D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  return 0;
}
static int zero_pair(nc_handle* h, FieldPair& f) {
  CU(cudaMemsetAsync(f.r, 0, h->D.npt * sizeof(double), h->stream));
  CU(cudaMemsetAsync(f.p, 0, h->D.npl * sizeof(double), h->stream));
  return h->prof ? mark(h, "lin_zero") : 0;
}
// the exchange adjoint on one field (k_comm_adj_add, then the destinations cleared)
static int comm_adj(nc_handle* h, FieldPair& f) {
  const long long ne = (long long)(h->nr + h->np) * h->D.KA;
  if (ne == 0) return 0;
  const unsigned g = (unsigned)((ne + 255) / 256);
  k_comm_adj_add<<<g, 256, 0, h->stream>>>(f.r, f.p, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
  TRY(check_launch(h, "comm_adj"));
  k_comm_adj_clear<<<g, 256, 0, h->stream>>>(f.r, f.p, h->r_dst, h->nr, h->p_dst, h->np);
  return check_launch(h, "comm_adj_clear");
}
static int vadv_lin_launch(nc_handle* h, int mode, const FieldPair& at, const FieldPair& den, const double* in_r,
                           const double* in_p, double* out_r, double* out_p, bool second) {
  for (int pole = 0; pole < 2; ++pole) {
    VadvLin a{pole ? at.p : at.r, pole ? den.p : den.r, pole ? h->flx_v.p : h->flx_v.r,
              pole ? h->frhog.p : h->frhog.r, pole ? in_p : in_r, pole ? out_p : out_r, h->dtl, 0.0,
              second ? 1 : 0, mode};
    const long long n = pole ? 6LL * h->D.LP : h->D.npt2;
    k_vadv_lin<<<(unsigned)((n + 63) / 64), 64, 0, h->stream>>>(a, pole);
    TRY(check_launch(h, mode == 1 ? "vadv_tl" : "vadv_ad"));
  }
  return 0;
}
static HLin hlin_args(nc_handle* h) {
  HLin a{};
  FieldPair* L = h->lin;
  a.q = h->q.r; a.Qmin = h->Qmin.r; a.Qmax = h->Qmax.r; a.rhog_t = L[LN_RHO].r; a.frhog = h->frhog.r;
  for (int f = 0; f < 3; ++f) a.qa[f] = h->qa[f].r;
  for (int f = 0; f < 6; ++f) { a.ch[f] = h->ch[f].r; a.cm[f] = h->cm[f].r; a.flx[f] = h->flx[f].r; }
  for (int f = 0; f < 9; ++f) a.xc[f] = h->xc[f].r;
  a.q_pl = h->q.p; a.qa_pl = h->qa[0].p; a.Qmin_pl = h->Qmin.p; a.Qmax_pl = h->Qmax.p; a.rhog_t_pl = L[LN_RHO].p;
  a.frhog_pl = h->frhog.p; a.ch_pl = h->ch[0].p; a.cm_pl = h->cm[0].p; a.flx_pl = h->flx[0].p; a.xc_pl = h->xc[0].p;
  a.dt = h->dtl;
  a.dq = L[LN_DQ].r; a.dq_pl = L[LN_DQ].p;
  for (int f = 0; f < 3; ++f) a.dqa[f] = L[LN_DQA0 + f].r;
  a.dqa_pl = L[LN_DQA0].p;
  a.dQmin = L[LN_DQN].r; a.dQmax = L[LN_DQX].r; a.dQmin_pl = L[LN_DQN].p; a.dQmax_pl = L[LN_DQX].p;
  a.oQmin = L[LN_DQN].r; a.oQmax = L[LN_DQX].r; a.oQmin_pl = L[LN_DQN].p; a.oQmax_pl = L[LN_DQX].p;
  a.gq = L[LN_DQ].r; a.gq_pl = L[LN_DQ].p;
  for (int f = 0; f < 3; ++f) a.gqa[f] = L[LN_DQA0 + f].r;
  a.gqa_pl = L[LN_DQA0].p;
  a.gQmin = L[LN_DQN].r; a.gQmax = L[LN_DQX].r; a.gQmin_pl = L[LN_DQN].p; a.gQmax_pl = L[LN_DQX].p;
  for (int d = 0; d < 3; ++d) { a.gg[d] = L[LN_DG0 + d].r; a.gg_pl[d] = L[LN_DG0 + d].p; }
  return a;
}

// the forward tracer step of x0 with the fluxes of the handle's last step,
// keeping its stages: X0 the input, X1 after the first vertical step, X2 after the
// horizontal step (and H's q, qa, Qmin / Qmax), X3 after the second
// vertical step; rhog_t before the horizontal update in LN_RHO
static int trc_lin_forward(nc_handle* h, const double* x0, const double* x0_pl) {
  FieldPair* L = h->lin;
  TRY(trc_vflux<double>(h));
  TRY(trc_hflux<double>(h));
  TRY(copy_in(h, L[LN_RHO], h->rhog_t.r, h->rhog_t.p));
  TRY(copy_in(h, L[LN_X0], x0, x0_pl));
  TRY(copy_in(h, L[LN_X1], x0, x0_pl));
  TRY(trc_vadv<double>(h, L[LN_X1], false));
  TRY(copy_in(h, L[LN_X2], L[LN_X1].r, L[LN_X1].p));
  TRY(trc_horizontal<double>(h, L[LN_X2]));
  TRY(trc_rhog<double>(h));
  TRY(copy_in(h, L[LN_X3], L[LN_X2].r, L[LN_X2].p));
  return trc_vadv<double>(h, L[LN_X3], true);
}

// tangent-linear of the horizontal step at X1: T2 = H'(X1) T1
static int hlin_tl(nc_handle* h) {
  const Dims& D = h->D;
  FieldPair* L = h->lin;
  const cudaStream_t s = h->stream;
  const unsigned pkb = (unsigned)((D.KA * D.LP + 127) / 128), cb = (unsigned)((D.npt2 + 127) / 128);
  {
    const dim3 gt((unsigned)D.KA, (unsigned)(((D.G - 2 + TG_DX - 1) / TG_DX) * ((D.G - 2 + TG_DY - 1) / TG_DY)),
                  (unsigned)D.L);
    k_trc_grad_t<<<gt, TG_DX * TG_DY, 0, s>>>(L[LN_T1].r, L[LN_RHO].r, L[LN_DQ].r, L[LN_DG0].r, L[LN_DG1].r,
                                              L[LN_DG2].r);
    TRY(check_launch(h, "lin_grad"));
  }
  k_trc_grad_pl<<<pkb, 128, 0, s>>>(L[LN_T1].p, L[LN_RHO].p, L[LN_DQ].p, L[LN_DG0].p, L[LN_DG1].p, L[LN_DG2].p);
  TRY(check_launch(h, "lin_grad_pl"));
  TRY(comm<double>(h, {L[LN_DG0], L[LN_DG1], L[LN_DG2]}));
  TrcRemapArgs<double> ra;
  ra.q = L[LN_DQ].r; ra.gq0 = L[LN_DG0].r; ra.gq1 = L[LN_DG1].r; ra.gq2 = L[LN_DG2].r;
  for (int f = 0; f < 9; ++f) ra.xc[f] = h->xc[f].r;
  for (int f = 0; f < 6; ++f) ra.cm[f] = h->cm[f].r;
  for (int f = 0; f < 3; ++f) ra.qa[f] = L[LN_DQA0 + f].r;
  k_trc_remap<<<cb, 128, 0, s>>>(ra);
  TRY(check_launch(h, "lin_remap"));
  TrcRemapPlArgs<double> rp;
  rp.q = L[LN_DQ].p; rp.gq0 = L[LN_DG0].p; rp.gq1 = L[LN_DG1].p; rp.gq2 = L[LN_DG2].p; rp.xc = h->xc[0].p;
  rp.cm = h->cm[0].p; rp.qa = L[LN_DQA0].p;
  k_trc_remap_pl<<<pkb, 128, 0, s>>>(rp);
  TRY(check_launch(h, "lin_remap_pl"));
  HLin a = hlin_args(h);
  k_hlin_qout<<<cb, 128, 0, s>>>(a, 0);
  TRY(check_launch(h, "lin_qout"));
  k_hlin_pole<<<pkb, 128, 0, s>>>(a, 0, 0);
  TRY(check_launch(h, "lin_qout_pl"));
  TRY(comm<double>(h, {L[LN_DQN], L[LN_DQX]}));
  a.x = L[LN_T1].r; a.x_pl = L[LN_T1].p; a.y = L[LN_T2].r; a.y_pl = L[LN_T2].p;
  k_hlin_apply<<<cb, 128, 0, s>>>(a, 0);
  TRY(check_launch(h, "lin_apply"));
  k_hlin_pole<<<pkb, 128, 0, s>>>(a, 0, 1);
  return check_launch(h, "lin_apply_pl");
}

// adjoint of the horizontal step at X1: T2 = H'(X1)^T T1
static int hlin_ad(nc_handle* h) {
  const Dims& D = h->D;
  FieldPair* L = h->lin;
  const cudaStream_t s = h->stream;
  const unsigned pkb = (unsigned)((D.KA * D.LP + 127) / 128), cb = (unsigned)((D.npt2 + 127) / 128);
  for (int n : {LN_DQ, LN_DG0, LN_DG1, LN_DG2, LN_DQA0, LN_DQA1, LN_DQA2, LN_DQN, LN_DQX}) TRY(zero_pair(h, L[n]));
  TRY(copy_in(h, L[LN_T2], L[LN_T1].r, L[LN_T1].p));   // y = x - ...: the direct part
  HLin a = hlin_args(h);
  a.x = L[LN_T1].r; a.x_pl = L[LN_T1].p;
  a.gx = L[LN_T2].r; a.gx_pl = L[LN_T2].p;
  k_hlin_apply<<<cb, 128, 0, s>>>(a, 1);
  TRY(check_launch(h, "lin_apply_ad"));
  k_hlin_pole<<<pkb, 128, 0, s>>>(a, 1, 1);
  TRY(check_launch(h, "lin_apply_ad_pl"));
  TRY(comm_adj(h, L[LN_DQN]));
  TRY(comm_adj(h, L[LN_DQX]));
  k_hlin_qout<<<cb, 128, 0, s>>>(a, 1);
  TRY(check_launch(h, "lin_qout_ad"));
  k_hlin_pole<<<pkb, 128, 0, s>>>(a, 1, 0);
  TRY(check_launch(h, "lin_qout_ad_pl"));
  k_hlin_remap_ad<<<cb, 128, 0, s>>>(a);
  TRY(check_launch(h, "lin_remap_ad"));
  k_hlin_pole_remap_ad<<<pkb, 128, 0, s>>>(a);
  TRY(check_launch(h, "lin_remap_ad_pl"));
  for (int d = 0; d < 3; ++d) TRY(comm_adj(h, L[LN_DG0 + d]));
  k_hlin_grad_ad<<<(unsigned)((D.npt + 255) / 256), 256, 0, s>>>(a);
  TRY(check_launch(h, "lin_grad_ad"));
  k_hlin_pole_grad_ad<<<pkb, 128, 0, s>>>(a);
  return check_launch(h, "lin_grad_ad_pl");
}

// lifts the pole kernels onto the library stream for the duration of a call
struct SingleStream {
  nc_handle* h;
  explicit SingleStream(nc_handle* hh) : h(hh) { h->single = true; }
  ~SingleStream() { h->single = false; }
};


// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
// the Held & Suarez (1994) parameters (nhm/forcing/mod_af_heldsuarez.py:19-39),
// with the moist case's equilibrium profile for DCMIP2016 case 2-1
static HsParams hs_params(const nc_handle* h, bool moist = false) {
  HsParams hp;
  hp.RdCp = h->C.Rdry / h->C.CPdry;
  hp.sigma_b = 0.7;
  hp.Kf = 1.0 / (1.0 * 86400.0);
  hp.Dth_z = 10.0;
  hp.Ka = 1.0 / (40.0 * 86400.0);
  hp.Ks = 1.0 / (4.0 * 86400.0);
  hp.T_eq0 = moist ? 294.0 : 315.0;
  hp.DT_y = moist ? 65.0 : 60.0;
  hp.PRE00 = h->C.PRE00;
  return hp;
}

extern "C" {

int nc_forcing_step(nc_handle* h) {
  if (!h) return fail(NC_ERR_ARG, "nc_forcing_step: null handle");
  TRY(f64_only(h, "nc_forcing_step"));
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_forcing_step: no state uploaded");
  if (!h->hs_lat && !h->kess_zf)
    return fail(NC_ERR_STATE, "nc_forcing_step: the handle was created without AF_hs_lat_terms or "
                              "AF_dcmip_kessler_zf (no forcing configured)");
  TRY(load_consts(h));
  const Dims& D = h->D;
  if (h->kess_zf) {
    DcmipArgs a;
    for (int v = 0; v < 6; ++v) a.P.v[v] = h->P[v].r;
    for (int n = 0; n < D.nq; ++n) a.Pq[n] = h->Pq[n].r;
    a.nq = D.nq;
    a.zf = h->kess_zf;
    a.precip = h->kess_precip;
    a.dt = h->dtl;
    a.RdCp = h->C.Rdry / h->C.CPdry;
    a.PRE00 = h->C.PRE00;
    a.negative_fixer = h->kess_negative_fixer;
    a.update_tot_dens = h->kess_update_tot_dens;
    a.n_cl = h->kess_n_cl;
    a.n_cl2 = h->kess_n_cl2;
    a.lat = h->kess_lat;
    a.lon = h->kess_lon;
    a.kessler = h->kess_on;
    a.sm = h->sm_on;
    a.sm_lsc = h->sm_lsc;
    a.sm_bryan = h->sm_bryan;
    a.zh = h->sm_zh;
    a.zsfc = h->sm_zsfc;
    a.tsurf = h->sm_tsurf;
    a.ij = h->sm_ij;
    a.hs = h->dcmip_hs;
    a.sm_C = h->dcmip_hs ? 0.0011 * 4.0 : 0.0011;   // simple_physics.py:25-46
    a.hs_lat3 = h->dcmip_hs_lat;
    a.hp = hs_params(h, true);
    k_forcing_dcmip<<<(unsigned)((D.npt2 + 63) / 64), 64, 0, h->stream>>>(a);
    TRY(check_launch(h, "forcing_dcmip"));
    TRY(comm_prg<double>(h));
    TRY(join_pl(h));
    return 0;
  }
  HsArgs a;
  for (int v = 0; v < 6; ++v) a.P.v[v] = h->P[v].r;
  for (int n = 0; n < h->C.nqw; ++n) a.Pqw[n] = h->Pq[n].r;
  a.lat3 = h->hs_lat;
  a.dt = h->dtl;
  a.hp = hs_params(h);
  k_forcing_hs<<<(unsigned)((D.npt2 + kBlock - 1) / kBlock), kBlock, 0, h->stream>>>(a);
  TRY(check_launch(h, "forcing_hs"));
  TRY(comm_prg<double>(h));
  TRY(join_pl(h));
  return 0;
}

int nc_forcing_precip(nc_handle* h, double* host) {
  if (!h || !host) return fail(NC_ERR_ARG, "nc_forcing_precip: null argument");
  if (!h->kess_precip) return fail(NC_ERR_STATE, "nc_forcing_precip: no Kessler forcing configured");
  TRY(load_consts(h));
  const Dims& D = h->D;
  CU(cudaStreamSynchronize(h->stream));
  std::vector<double> tmp((size_t)D.L * D.G * D.G);
  CU(cudaMemcpy(tmp.data(), h->kess_precip, tmp.size() * sizeof(double), cudaMemcpyDeviceToHost));
  for (int l = 0; l < D.L; ++l)
    for (int j = 0; j < D.G; ++j)
      for (int i = 0; i < D.G; ++i) host[((size_t)i * D.G + j) * D.L + l] = tmp[((size_t)l * D.G + j) * D.G + i];
  return 0;
}

const char* nc_last_error(void) { return g_err.c_str(); }

int64_t nc_kernel_launches(nc_handle* h) { return h ? h->launches : 0; }

// float32 copy of n float64 device values
__global__ void k_to_f32(const double* src, float* dst, long long n) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) dst[t] = (float)src[t];
}
static int to_f32(nc_handle* h, const double* src, long long n, const float** dst) {
  if (!src) {
    *dst = nullptr;
    return 0;
  }
  float* d = nullptr;
  TRY(dev_alloc_bytes(h, (void**)&d, (size_t)n * sizeof(float)));
  k_to_f32<<<(unsigned)((n + 255) / 256), 256>>>(src, d, n);
  CU(cudaGetLastError());
  *dst = d;
  return 0;
}

// The mixed form's float32 geometry and constants, rounded from the float64
// ones (which stay resident: the mass sums read GSGAM2 in float64).
static int make_f32_geometry(nc_handle* h) {
  const Dims& D = h->D;
  const Geom& G = h->Gm;
  GeomT<float>& F = h->Gmf;
  const long long n3 = D.npt, n2 = D.npt2, np = D.npl, gl = 6LL * D.LP;
  struct Item {
    const double* src;
    long long n;
    const float** dst;
  } items[] = {
      {G.GSGAM2, n3, &F.GSGAM2}, {G.GSGAM2H, n3, &F.GSGAM2H}, {G.RGSGAM2, n3, &F.RGSGAM2},
      {G.RGSGAM2H, n3, &F.RGSGAM2H}, {G.RGSQRTH, n3, &F.RGSQRTH}, {G.RGAM, n3, &F.RGAM}, {G.RGAMH, n3, &F.RGAMH},
      {G.GAM2H, n3, &F.GAM2H}, {G.PHI, n3, &F.PHI}, {G.C2W, 2 * n3, &F.C2W}, {G.W2C, 2 * n3, &F.W2C},
      {G.C2WGz, 6 * n3, &F.C2WGz}, {G.rho_bs, n3, &F.rho_bs}, {G.pre_bs, n3, &F.pre_bs}, {G.tem_bs, n3, &F.tem_bs},
      {G.coef_div, 21 * n2, &F.coef_div}, {G.coef_grad, 21 * n2, &F.coef_grad}, {G.coef_lap, 7 * n2, &F.coef_lap},
      {G.coef_intp, 18 * n2, &F.coef_intp}, {G.intp_w, 18 * n2, &F.intp_w}, {G.coef_diff, 18 * n2, &F.coef_diff},
      {G.GRD_x, 3 * n2, &F.GRD_x}, {G.GRD_xr, 9 * n2, &F.GRD_xr}, {G.GMTR_t, 6 * n2, &F.GMTR_t},
      {G.GMTR_a, 9 * n2, &F.GMTR_a}, {G.GMTR_p, n2, &F.GMTR_p},
      {G.GSGAM2_pl, np, &F.GSGAM2_pl}, {G.GSGAM2H_pl, np, &F.GSGAM2H_pl}, {G.RGSGAM2_pl, np, &F.RGSGAM2_pl},
      {G.RGSGAM2H_pl, np, &F.RGSGAM2H_pl}, {G.RGSQRTH_pl, np, &F.RGSQRTH_pl}, {G.RGAM_pl, np, &F.RGAM_pl},
      {G.RGAMH_pl, np, &F.RGAMH_pl}, {G.GAM2H_pl, np, &F.GAM2H_pl}, {G.PHI_pl, np, &F.PHI_pl},
      {G.C2W_pl, 2 * np, &F.C2W_pl}, {G.W2C_pl, 2 * np, &F.W2C_pl}, {G.C2WGz_pl, 6 * np, &F.C2WGz_pl},
      {G.rho_bs_pl, np, &F.rho_bs_pl}, {G.pre_bs_pl, np, &F.pre_bs_pl}, {G.tem_bs_pl, np, &F.tem_bs_pl},
      {G.coef_div_pl, gl * 3, &F.coef_div_pl}, {G.coef_grad_pl, gl * 3, &F.coef_grad_pl},
      {G.coef_lap_pl, gl, &F.coef_lap_pl}, {G.coef_intp_pl, gl * 9, &F.coef_intp_pl},
      {G.coef_diff_pl, gl * 3, &F.coef_diff_pl}, {G.GRD_x_pl, gl * 3, &F.GRD_x_pl}, {G.GRD_xr_pl, gl * 3, &F.GRD_xr_pl},
      {G.GMTR_t_pl, gl * 5, &F.GMTR_t_pl}, {G.GMTR_a_pl, gl * 18, &F.GMTR_a_pl}, {G.GMTR_p_pl, gl * 8, &F.GMTR_p_pl},
  };
  for (const Item& it : items) TRY(to_f32(h, it.src, it.n, it.dst));
  F.pntmask = G.pntmask;
  F.have_sgp = G.have_sgp;
  CU(cudaDeviceSynchronize());
  const Consts& C = h->C;
  ConstsT<float>& Cf = h->Cf;
  Cf.GRAV = (float)C.GRAV; Cf.Rdry = (float)C.Rdry; Cf.CVdry = (float)C.CVdry; Cf.CPdry = (float)C.CPdry;
  Cf.Rvap = (float)C.Rvap; Cf.OHM = (float)C.OHM;
  // the reference's float32 constants (share/mod_const.py:170-172): EPS and HUGE are
  // the working type's machine epsilon and largest value (the float64 HUGE would
  // round to infinity, and 0 * HUGE in the limiters' masks would give NaN)
  Cf.EPS = FLT_EPSILON;
  Cf.HUGE_ = FLT_MAX;
  Cf.rscale = (float)C.rscale; Cf.alpha = (float)C.alpha; Cf.Kh = (float)C.Kh; Cf.divdamp_coef = (float)C.divdamp_coef;
  Cf.hdiff_fact_rho = (float)C.hdiff_fact_rho; Cf.CVW0 = (float)C.CVW0; Cf.PRE00 = (float)C.PRE00;
  for (int n = 0; n < NC_MAXQW; ++n) Cf.CVW[n] = (float)C.CVW[n];
  Cf.nqw = C.nqw;
  Cf.hdiff_nl = C.hdiff_nl; Cf.nl_c1 = (float)C.nl_c1; Cf.nl_area = (float)C.nl_area; Cf.nl_min = (float)C.nl_min;
  Cf.rayleigh = C.rayleigh; Cf.rayleigh_only_w = C.rayleigh_only_w;
  Cf.gam_unit = C.gam_unit;
  Cf.rsc_h = (float)(1.0 / C.rscale);   // the float32 divisions multiply by the rounded reciprocal
  Cf.rsc_l = 0.0f;
  Cf.third_h = (float)(1.0 / 3.0);
  Cf.third_l = 0.0f;
  for (int k = 0; k < NC_MAXK; ++k) {
    Cf.afact[k] = (float)C.afact[k]; Cf.bfact[k] = (float)C.bfact[k]; Cf.cfact[k] = (float)C.cfact[k];
    Cf.dfact[k] = (float)C.dfact[k]; Cf.rdgz[k] = (float)C.rdgz[k]; Cf.rdgzh[k] = (float)C.rdgzh[k];
    Cf.nl_khmax[k] = (float)C.nl_khmax[k]; Cf.ray_c[k] = (float)C.ray_c[k]; Cf.ray_ch[k] = (float)C.ray_ch[k];
  }
  return 0;
}

static int create_impl(const nc_array* arrays, int32_t narrays, nc_handle* h) {
  // the multi-level hyperdiffusion kernel takes more than the default 48 KB of
  // dynamic shared memory in its float64 instance
  CU(cudaFuncSetAttribute(k_hdiff2_m<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, hdiff2_m_smem<double>()));
  CU(cudaFuncSetAttribute(k_hdiff2_m<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, hdiff2_m_smem<float>()));
  CU(cudaFuncSetAttribute(k_dd3d_m<double, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dd3d_m_smem<double>()));
  CU(cudaFuncSetAttribute(k_dd3d_m<float, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, dd3d_m_smem<float>()));
  ArrTab T;
  for (int n = 0; n < narrays; ++n) {
    if (!arrays[n].name || !arrays[n].data) return fail(NC_ERR_ARG, "null array entry");
    T.m[arrays[n].name] = &arrays[n];
  }
  double v;
  Dims& D = h->D;
  TRY(scalar(T, "gall_1d", v)); D.G = (int)v;
  TRY(scalar(T, "kall", v)); D.KA = (int)v;
  TRY(scalar(T, "lall", v)); D.L = (int)v;
  TRY(scalar(T, "kmin", v)); D.kmin = (int)v;
  TRY(scalar(T, "kmax", v)); D.kmax = (int)v;
  TRY(scalar(T, "gmin", v)); D.gmin = (int)v;
  TRY(scalar(T, "gmax", v)); D.gmax = (int)v;
  TRY(scalar(T, "nq", v)); D.nq = (int)v;
  D.LP = 2;
  if (T.get("members")) {   // ensemble members stacked along the region axis (lall = 40 * members)
    double mem;
    TRY(scalar(T, "members", mem));
    if (mem < 1 || mem > 4096) return fail(NC_ERR_ARG, "members must be 1..4096");
    D.LP = 2 * (int)mem;
  }
  if (D.G < 4 || D.KA < 4 || D.KA > NC_MAXK || D.L < 1 || D.kmin != 1 || D.kmax != D.KA - 2 || D.gmin != 1 ||
      D.gmax != D.G - 2 || D.nq < 1 || D.nq > NC_MAXNQ)
    return fail(NC_ERR_ARG, "unsupported grid dimensions (need kmin=1, kmax=kall-2, 1<=nq<=32, kall<=128)");
  D.plane = (long long)D.G * D.G;
  D.npt = D.plane * D.KA * D.L;
  D.npt2 = D.plane * D.L;
  D.npl = 6 * D.KA * D.LP;
  if (D.npt * 6 > 2147483647LL)
    return fail(NC_ERR_ARG, "grid too large for 32-bit device indexing (6 * lall * kall * gall_1d^2 >= 2^31)");
  D.planei = (int)D.plane;
  D.npti = (int)D.npt;
  D.npt2i = (int)D.npt2;
  Consts& C = h->C;
  TRY(scalar(T, "GRAV", C.GRAV)); TRY(scalar(T, "Rdry", C.Rdry)); TRY(scalar(T, "CVdry", C.CVdry));
  TRY(scalar(T, "CPdry", C.CPdry)); TRY(scalar(T, "Rvap", C.Rvap)); TRY(scalar(T, "OHM", C.OHM));
  TRY(scalar(T, "EPS", C.EPS)); TRY(scalar(T, "HUGE", C.HUGE_)); TRY(scalar(T, "rscale", C.rscale));
  TRY(scalar(T, "alpha", C.alpha)); TRY(scalar(T, "Kh_coef", C.Kh)); TRY(scalar(T, "divdamp_coef", C.divdamp_coef));
  TRY(scalar(T, "hdiff_fact_rho", C.hdiff_fact_rho));
  if (!(C.rscale != 0.0 && std::isfinite(C.rscale))) return fail(NC_ERR_ARG, "rscale must be finite and nonzero");
  if (T.get("precision")) {   // 0: float64, 1: mixed (float32 bulk, float64 HEVI solve / deviations / sums)
    double pr;
    TRY(scalar(T, "precision", pr));
    if (pr != 0.0 && pr != 1.0) return fail(NC_ERR_ARG, "precision must be 0 (float64) or 1 (mixed)");
    h->mixed = (pr == 1.0);
  }
  recip_pair(C.rscale, C.rsc_h, C.rsc_l);
  recip_pair(3.0, C.third_h, C.third_l);
  TRY(scalar(T, "dtl", h->dtl)); TRY(scalar(T, "dts", h->dts));
  {
    const nc_array* cvw = T.get("CVW");
    if (!cvw || cvw->dtype != NC_F64 || numel(cvw) < 1) return fail(NC_ERR_ARG, "missing CVW");
    C.CVW0 = ((const double*)cvw->data)[0];
    // water tracers 0..NQW_END (optional entry; one, the vapour, when absent)
    C.nqw = 1;
    if (T.get("NQW_END")) {
      double f;
      TRY(scalar(T, "NQW_END", f));
      C.nqw = (int)f + 1;
    }
    if (C.nqw < 1 || C.nqw > NC_MAXQW || C.nqw > numel(cvw) || C.nqw > D.nq)
      return fail(NC_ERR_ARG, "NQW_END must give 1.." + std::to_string(NC_MAXQW) +
                                  " water tracers among the nq tracers, with CVW for each");
    for (int n = 0; n < NC_MAXQW; ++n) C.CVW[n] = n < C.nqw ? ((const double*)cvw->data)[n] : 0.0;
    if (T.get("trcadv")) {
      double f;
      TRY(scalar(T, "trcadv", f));   // 1: DCMIP 1-1 winds, 2: DCMIP 1-2 winds
      if (f != 0.0 && f != 1.0 && f != 2.0) return fail(NC_ERR_ARG, "trcadv must be 0, 1 (DCMIP 1-1) or 2 (1-2)");
      h->trcadv = (f != 0.0);
      h->trcadv_hadley = (f == 2.0);
    }
    const nc_array* ss = T.get("sstep");
    if (!ss || numel(ss) > 4 || (numel(ss) < 1 && !h->trcadv)) return fail(NC_ERR_ARG, "missing sstep");
    h->nstage = (int)numel(ss);
    for (int n = 0; n < h->nstage; ++n) {
      h->sstep[n] = (ss->dtype == NC_I64) ? (int)((const int64_t*)ss->data)[n] : (int)((const int32_t*)ss->data)[n];
      if (h->sstep[n] < 1) return fail(NC_ERR_ARG, "sstep entries must be >= 1");
    }
  }
  TRY(up_vec(T, "GRD_afact", D.KA, C.afact)); TRY(up_vec(T, "GRD_bfact", D.KA, C.bfact));
  TRY(up_vec(T, "GRD_cfact", D.KA, C.cfact)); TRY(up_vec(T, "GRD_dfact", D.KA, C.dfact));
  TRY(up_vec(T, "GRD_rdgz", D.KA, C.rdgz)); TRY(up_vec(T, "GRD_rdgzh", D.KA, C.rdgzh));
  if (T.get("hdiff_nl_kh_max")) {   // hyperdiffusion NONLINEAR1 (mod_numfilter.py:1153-1206)
    C.hdiff_nl = 1;
    TRY(up_vec(T, "hdiff_nl_kh_max", D.KA, C.nl_khmax));
    TRY(scalar(T, "hdiff_nl_c1", C.nl_c1));
    TRY(scalar(T, "hdiff_nl_area", C.nl_area));
    TRY(scalar(T, "hdiff_nl_minlim", C.nl_min));
  }
  if (T.get("rayleigh_coef")) {   // Rayleigh sponge (mod_numfilter.py:219-271)
    C.rayleigh = 1;
    TRY(up_vec(T, "rayleigh_coef", D.KA, C.ray_c));
    TRY(up_vec(T, "rayleigh_coef_h", D.KA, C.ray_ch));
    if (T.get("rayleigh_only_w")) {
      double f;
      TRY(scalar(T, "rayleigh_only_w", f));
      C.rayleigh_only_w = (f != 0.0);
    }
  }
  Geom& Gm = h->Gm;
  const int KA = D.KA;
  TRY(up_reg(h, T, "VMTR_GSGAM2", KA, 1, &Gm.GSGAM2));
  TRY(up_reg(h, T, "VMTR_GSGAM2H", KA, 1, &Gm.GSGAM2H));
  TRY(up_reg(h, T, "VMTR_RGSGAM2", KA, 1, &Gm.RGSGAM2));
  TRY(up_reg(h, T, "VMTR_RGSGAM2H", KA, 1, &Gm.RGSGAM2H));
  TRY(up_reg(h, T, "VMTR_RGSQRTH", KA, 1, &Gm.RGSQRTH));
  TRY(up_reg(h, T, "VMTR_RGAM", KA, 1, &Gm.RGAM));
  TRY(up_reg(h, T, "VMTR_RGAMH", KA, 1, &Gm.RGAMH));
  TRY(up_reg(h, T, "VMTR_GAM2H", KA, 1, &Gm.GAM2H));
  TRY(up_reg(h, T, "VMTR_PHI", KA, 1, &Gm.PHI));
  TRY(up_reg(h, T, "VMTR_C2Wfact", KA, 2, &Gm.C2W));
  TRY(up_reg(h, T, "VMTR_W2Cfact", KA, 2, &Gm.W2C));
  TRY(up_reg(h, T, "VMTR_C2WfactGz", KA, 6, &Gm.C2WGz));
  TRY(up_reg(h, T, "rho_bs", KA, 1, &Gm.rho_bs));
  TRY(up_reg(h, T, "pre_bs", KA, 1, &Gm.pre_bs));
  TRY(up_reg(h, T, "tem_bs", KA, 1, &Gm.tem_bs));
  {
    const double* vol;
    TRY(up_reg(h, T, "VMTR_VOLUME", KA, 1, &vol));
    h->vol = const_cast<double*>(vol);
  }
  TRY(up_reg(h, T, "OPRT_coef_div", 1, 21, &Gm.coef_div));
  TRY(up_reg(h, T, "OPRT_coef_grad", 1, 21, &Gm.coef_grad));
  TRY(up_reg(h, T, "OPRT_coef_lap", 1, 7, &Gm.coef_lap));
  TRY(up_reg(h, T, "OPRT_coef_intp", 1, 18, &Gm.coef_intp));
  {
    double* w;
    TRY(dev_alloc(h, &w, (size_t)18 * D.npt2));
    k_intp_weights<<<(unsigned)((D.npt2 + 255) / 256), 256>>>(Gm.coef_intp, w, (int)D.npt2);
    CU(cudaGetLastError());
    CU(cudaDeviceSynchronize());
    Gm.intp_w = w;
  }
  TRY(up_reg(h, T, "OPRT_coef_diff", 1, 18, &Gm.coef_diff));
  TRY(up_reg(h, T, "GRD_x", 1, 3, &Gm.GRD_x));
  TRY(up_reg(h, T, "GRD_xr", 1, 9, &Gm.GRD_xr));
  TRY(up_reg(h, T, "GMTR_t_W", 1, 6, &Gm.GMTR_t));
  TRY(up_reg(h, T, "GMTR_a_HN", 1, 9, &Gm.GMTR_a));
  TRY(up_reg(h, T, "GMTR_p_RAREA", 1, 1, &Gm.GMTR_p));
  {
    // shallow atmosphere: every gamma factor exactly 1 (checked element by element)
    bool unit = true;
    for (const char* nm : {"VMTR_RGAM", "VMTR_RGAMH", "VMTR_GAM2H", "VMTR_RGAM_pl", "VMTR_RGAMH_pl", "VMTR_GAM2H_pl"}) {
      const nc_array* a = T.get(nm);
      if (!a || a->dtype != NC_F64) { unit = false; break; }
      const double* d = (const double*)a->data;
      for (int64_t n = 0, e = numel(a); n < e && unit; ++n) unit = (d[n] == 1.0);
    }
    C.gam_unit = unit ? 1 : 0;
  }
  if (h->trcadv) {   // the coordinates the prescribed winds are computed from
    TRY(up_reg(h, T, "GRD_LON", 1, 1, &h->trc_lon));
    TRY(up_reg(h, T, "GRD_LAT", 1, 1, &h->trc_lat));
    TRY(up_reg(h, T, "GRD_Z", KA, 1, &h->trc_zf));
    TRY(up_reg(h, T, "GRD_ZH", KA, 1, &h->trc_zh));
    TRY(up_pl(h, T, "GRD_LON_pl", 6LL * D.LP, &h->trc_lon_pl));
    TRY(up_pl(h, T, "GRD_LAT_pl", 6LL * D.LP, &h->trc_lat_pl));
    TRY(up_pl(h, T, "GRD_Z_pl", D.npl, &h->trc_zf_pl));
    TRY(up_pl(h, T, "GRD_ZH_pl", D.npl, &h->trc_zh_pl));
    TRY(dev_alloc(h, &h->trc_time, 1));
    CU(cudaMemset(h->trc_time, 0, sizeof(double)));
  }
  if (T.get("AF_dcmip_kessler_zf")) {   // DCMIP forcing (nc_forcing_step): Kessler and / or simple physics
    if (T.get("AF_hs_lat_terms")) return fail(NC_ERR_ARG, "Held-Suarez and DCMIP forcing set-ups both given");
    if (!T.get("PRE00")) return fail(NC_ERR_ARG, "AF_dcmip_kessler_zf given without PRE00");
    if (C.nqw != 3 && C.nqw != 1)
      return fail(NC_ERR_ARG, "DCMIP forcing needs RAIN_TYPE WARM (NQW_END = 2: vapour, cloud, rain) or DRY");
    if (D.kmax - D.kmin + 1 > NC_KESS_K || D.kmax - D.kmin < 1)
      return fail(NC_ERR_ARG, "DCMIP forcing: 2.." + std::to_string(NC_KESS_K) + " model levels");
    if (const nc_array* sc = T.get("AF_dcmip_schemes")) {
      // [Kessler, simple physics, condensation(, Held-Suarez(, Bryan boundary layer))]
      if (sc->dtype != NC_I64 || numel(sc) < 3 || numel(sc) > 5)
        return fail(NC_ERR_ARG, "AF_dcmip_schemes: three to five int64 switches");
      const long long* f3 = (const long long*)sc->data;
      h->kess_on = f3[0] != 0;
      h->sm_on = f3[1] != 0;
      h->sm_lsc = h->sm_on && f3[2] != 0;
      h->dcmip_hs = numel(sc) >= 4 && f3[3] != 0;
      h->sm_bryan = h->sm_on && numel(sc) >= 5 && f3[4] != 0;
      if (!h->kess_on && !h->sm_on) return fail(NC_ERR_ARG, "AF_dcmip_schemes: neither Kessler nor simple physics");
    }
    if (h->kess_on && C.nqw != 3) return fail(NC_ERR_ARG, "Kessler microphysics needs RAIN_TYPE WARM");
    if (h->dcmip_hs) TRY(up_reg(h, T, "AF_dcmip_hs_lat_terms", 1, 3, &h->dcmip_hs_lat));
    if (h->sm_on) {   // what the simple physics reads besides the state (mod_forcing.py:236-250)
      TRY(up_reg(h, T, "AF_dcmip_zh", D.KA, 1, &h->sm_zh));
      TRY(up_reg(h, T, "AF_dcmip_zsfc", 1, 1, &h->sm_zsfc));
      TRY(up_reg(h, T, "AF_dcmip_tsurf", 1, 1, &h->sm_tsurf));
      TRY(up_reg(h, T, "AF_dcmip_ij", 1, 6, &h->sm_ij));
    }
    TRY(scalar(T, "PRE00", C.PRE00));
    TRY(up_reg(h, T, "AF_dcmip_kessler_zf", D.KA, 1, &h->kess_zf));
    double f;
    if (T.get("AF_negative_fixer")) {
      TRY(scalar(T, "AF_negative_fixer", f));
      h->kess_negative_fixer = f != 0.0;
    }
    if (T.get("AF_update_tot_dens")) {
      TRY(scalar(T, "AF_update_tot_dens", f));
      h->kess_update_tot_dens = f != 0.0;
    }
    TRY(dev_alloc(h, &h->kess_precip, (size_t)D.L * D.G * D.G));
    if (T.get("AF_dcmip_chem")) {   // the terminator toy chemistry on tracers (Cl, Cl2)
      const nc_array* ch = T.get("AF_dcmip_chem");
      if (ch->dtype != NC_I64 || numel(ch) != 2) return fail(NC_ERR_ARG, "AF_dcmip_chem: two int64 tracer indices");
      const long long* ix2 = (const long long*)ch->data;
      if (ix2[0] < C.nqw || ix2[1] < C.nqw || ix2[0] >= D.nq || ix2[1] >= D.nq || ix2[0] == ix2[1])
        return fail(NC_ERR_ARG, "AF_dcmip_chem: indices of two distinct non-water tracers");
      h->kess_n_cl = (int)ix2[0];
      h->kess_n_cl2 = (int)ix2[1];
      TRY(up_reg(h, T, "AF_dcmip_lat", 1, 1, &h->kess_lat));
      TRY(up_reg(h, T, "AF_dcmip_lon", 1, 1, &h->kess_lon));
    }
  }
  if (T.get("AF_hs_lat_terms")) {   // Held-Suarez forcing configured (nc_forcing_step)
    if (!T.get("PRE00")) return fail(NC_ERR_ARG, "AF_hs_lat_terms given without PRE00");
    TRY(scalar(T, "PRE00", C.PRE00));
    TRY(up_reg(h, T, "AF_hs_lat_terms", 1, 3, &h->hs_lat));
  }
  if (T.get("HIST_hgt")) {   // derived history diagnostics configured (nc_history_vars)
    if (!T.get("PRE00")) return fail(NC_ERR_ARG, "HIST_hgt given without PRE00");
    TRY(scalar(T, "PRE00", C.PRE00));
    TRY(up_reg(h, T, "HIST_hgt", D.KA, 1, &h->hist_hgt));
    TRY(up_reg(h, T, "HIST_coslat", 1, 1, &h->hist_coslat));
    TRY(up_reg(h, T, "HIST_zsfc", 1, 1, &h->hist_zsfc));
    TRY(up_reg(h, T, "HIST_area", 1, 1, &h->hist_area));
    TRY(up_reg(h, T, "HIST_IJ", 1, 6, &h->hist_IJ));
    TRY(up_pl(h, T, "HIST_dgz", D.KA, &h->hist_dgz));
    TRY(up_vec(T, "HIST_consts", 10, h->hist_c));
    const nc_array* tr = T.get("HIST_tracers");
    if (!tr || tr->dtype != NC_I64 || numel(tr) != 6) return fail(NC_ERR_ARG, "HIST_tracers: six int64 indices");
    for (int n = 0; n < 6; ++n) {
      const int64_t v = ((const int64_t*)tr->data)[n];
      if (v < -1 || v >= D.nq) return fail(NC_ERR_ARG, "HIST_tracers: index outside the tracers");
      h->hist_trc[n] = (int)v;
    }
    if (const nc_array* ch = T.get("HIST_chem")) {   // AF_TYPE 'DCMIP' with the terminator chemistry
      if (ch->dtype != NC_I64 || numel(ch) != 2) return fail(NC_ERR_ARG, "HIST_chem: two int64 tracer indices");
      for (int n = 0; n < 2; ++n) {
        const int64_t v = ((const int64_t*)ch->data)[n];
        if (v < 0 || v >= D.nq) return fail(NC_ERR_ARG, "HIST_chem: index outside the tracers");
        h->hist_chem[n] = (int)v;
      }
    }
    TRY(dev_alloc(h, &h->hist_thmean, (size_t)D.KA));
    h->hist = true;
  }
  const int64_t npl = D.npl;
  TRY(up_pl(h, T, "VMTR_GSGAM2_pl", npl, &Gm.GSGAM2_pl));
  TRY(up_pl(h, T, "VMTR_GSGAM2H_pl", npl, &Gm.GSGAM2H_pl));
  TRY(up_pl(h, T, "VMTR_RGSGAM2_pl", npl, &Gm.RGSGAM2_pl));
  TRY(up_pl(h, T, "VMTR_RGSGAM2H_pl", npl, &Gm.RGSGAM2H_pl));
  TRY(up_pl(h, T, "VMTR_RGSQRTH_pl", npl, &Gm.RGSQRTH_pl));
  TRY(up_pl(h, T, "VMTR_RGAM_pl", npl, &Gm.RGAM_pl));
  TRY(up_pl(h, T, "VMTR_RGAMH_pl", npl, &Gm.RGAMH_pl));
  TRY(up_pl(h, T, "VMTR_GAM2H_pl", npl, &Gm.GAM2H_pl));
  TRY(up_pl(h, T, "VMTR_PHI_pl", npl, &Gm.PHI_pl));
  TRY(up_pl(h, T, "VMTR_C2Wfact_pl", npl * 2, &Gm.C2W_pl));
  TRY(up_pl(h, T, "VMTR_W2Cfact_pl", npl * 2, &Gm.W2C_pl));
  TRY(up_pl(h, T, "VMTR_C2WfactGz_pl", npl * 6, &Gm.C2WGz_pl));
  TRY(up_pl(h, T, "rho_bs_pl", npl, &Gm.rho_bs_pl));
  TRY(up_pl(h, T, "pre_bs_pl", npl, &Gm.pre_bs_pl));
  TRY(up_pl(h, T, "tem_bs_pl", npl, &Gm.tem_bs_pl));
  {
    const double* vp;
    TRY(up_pl(h, T, "VMTR_VOLUME_pl", npl, &vp));
    h->vol_pl = const_cast<double*>(vp);
  }
  const int64_t gl = 6 * D.LP;
  TRY(up_pl(h, T, "OPRT_coef_div_pl", gl * 3, &Gm.coef_div_pl));
  TRY(up_pl(h, T, "OPRT_coef_grad_pl", gl * 3, &Gm.coef_grad_pl));
  TRY(up_pl(h, T, "OPRT_coef_lap_pl", gl, &Gm.coef_lap_pl));
  TRY(up_pl(h, T, "OPRT_coef_intp_pl", gl * 9, &Gm.coef_intp_pl));
  TRY(up_pl(h, T, "OPRT_coef_diff_pl", gl * 3, &Gm.coef_diff_pl));
  TRY(up_pl(h, T, "GRD_x_pl", gl * 3, &Gm.GRD_x_pl));
  TRY(up_pl(h, T, "GRD_xr_pl", gl * 3, &Gm.GRD_xr_pl));
  TRY(up_pl(h, T, "GMTR_t_pl", gl * 5, &Gm.GMTR_t_pl));
  TRY(up_pl(h, T, "GMTR_a_pl", gl * 18, &Gm.GMTR_a_pl));
  TRY(up_pl(h, T, "GMTR_p_pl", gl * 8, &Gm.GMTR_p_pl));
  // integer tables
  {
    const nc_array* pm = T.get("pntmask");
    if (!pm || numel(pm) != 2LL * D.L || (pm->dtype != NC_I32 && pm->dtype != NC_I64))
      return fail(NC_ERR_ARG, "bad pntmask");
    std::vector<int> tmp(2 * D.L);
    for (int n = 0; n < 2 * D.L; ++n)
      tmp[n] = pm->dtype == NC_I32 ? ((const int32_t*)pm->data)[n] : (int)((const int64_t*)pm->data)[n];
    int* dp;
    CU(cudaMalloc((void**)&dp, tmp.size() * sizeof(int)));
    h->allocs.push_back(dp);
    CU(cudaMemcpy(dp, tmp.data(), tmp.size() * sizeof(int), cudaMemcpyHostToDevice));
    Gm.pntmask = dp;
    const nc_array* sg = T.get("have_sgp");
    if (!sg || numel(sg) != D.L) return fail(NC_ERR_ARG, "bad have_sgp");
    std::vector<int> t2(D.L);
    for (int n = 0; n < D.L; ++n)
      t2[n] = sg->dtype == NC_BOOL ? ((const uint8_t*)sg->data)[n]
                                   : (sg->dtype == NC_I32 ? ((const int32_t*)sg->data)[n] : (int)((const int64_t*)sg->data)[n]);
    CU(cudaMalloc((void**)&dp, t2.size() * sizeof(int)));
    h->allocs.push_back(dp);
    CU(cudaMemcpy(dp, t2.data(), t2.size() * sizeof(int), cudaMemcpyHostToDevice));
    Gm.have_sgp = dp;
  }
  // halo plan
  {
    const nc_array* a = T.get("halo_r_dst");
    const nc_array* b = T.get("halo_r_src");
    const nc_array* c = T.get("halo_p_dst");
    const nc_array* d = T.get("halo_p_src");
    if (!a || !b || !c || !d || a->dtype != NC_I64 || b->dtype != NC_I64 || c->dtype != NC_I64 || d->dtype != NC_I64 ||
        numel(a) != numel(b) || numel(c) != numel(d))
      return fail(NC_ERR_ARG, "bad halo plan");
    h->nr = (int)numel(a);
    h->np = (int)numel(c);
    const nc_array* src[4] = {a, b, c, d};
    long long** dst[4] = {&h->r_dst, &h->r_src, &h->p_dst, &h->p_src};
    for (int n = 0; n < 4; ++n) {
      size_t bytes = (size_t)std::max<int64_t>(numel(src[n]), 1) * sizeof(long long);
      CU(cudaMalloc((void**)dst[n], bytes));
      h->allocs.push_back(*dst[n]);
      if (numel(src[n])) CU(cudaMemcpy(*dst[n], src[n]->data, numel(src[n]) * sizeof(long long), cudaMemcpyHostToDevice));
    }
  }
  if (h->mixed) {
    if (h->hist || h->hs_lat || h->kess_zf)
      return fail(NC_ERR_ARG, "the mixed-precision form runs the dynamics step and the offline tracer advection "
                              "only (no Held-Suarez forcing or history diagnostics set-up)");
    TRY(make_f32_geometry(h));
  }
  // state and work fields
  char nm[32];
  const char* pn[6] = {"RHOG", "RHOGVX", "RHOGVY", "RHOGVZ", "RHOGW", "RHOGE"};
  for (int v = 0; v < 6; ++v) TRY(field(h, h->P[v], pn[v]));
  for (int v = 0; v < D.nq; ++v) { snprintf(nm, sizeof nm, "RHOGQ.%d", v); TRY(field(h, h->Pq[v], nm)); }
  for (int v = 0; v < 6; ++v) { snprintf(nm, sizeof nm, "PROG0.%d", v); TRY(field(h, h->P0[v], nm)); }
  TRY(field(h, h->pre, "pre")); TRY(field(h, h->tem, "tem")); TRY(field(h, h->vx, "vx")); TRY(field(h, h->vy, "vy"));
  TRY(field(h, h->vz, "vz")); TRY(field(h, h->w, "w")); TRY(field(h, h->rho, "rho")); TRY(field(h, h->ein, "ein"));
  TRY(field(h, h->eth, "eth")); TRY(field(h, h->pregd, "pregd", true)); TRY(field(h, h->rhogd, "rhogd", true));
  for (int d = 0; d < 3; ++d) { snprintf(nm, sizeof nm, "vv.%d", d); TRY(field(h, h->vv[d], nm)); }
  for (int d = 0; d < 4; ++d) { snprintf(nm, sizeof nm, "gadv.%d", d); TRY(field(h, h->gadv[d], nm)); }
  for (int n = 0; n < 6; ++n) {
    snprintf(nm, sizeof nm, "vt.%d", n); TRY(field(h, h->vt[n], nm));
    snprintf(nm, sizeof nm, "vt2.%d", n); TRY(field(h, h->vt2[n], nm));
    snprintf(nm, sizeof nm, "gT0.%d", n); TRY(field(h, h->gT0[n], nm));
    snprintf(nm, sizeof nm, "gT.%d", n); TRY(field(h, h->gT[n], nm));
    snprintf(nm, sizeof nm, "PSa.%d", n); TRY(field(h, h->PSa[n], nm));
    snprintf(nm, sizeof nm, "PSb.%d", n); TRY(field(h, h->PSb[n], nm));
  }
  TRY(field(h, h->frhog, "frhog"));
  for (int n = 0; n < 5; ++n) { snprintf(nm, sizeof nm, "PM.%d", n); TRY(field(h, h->PM[n], nm)); }
  for (int d = 0; d < 3; ++d) {
    snprintf(nm, sizeof nm, "vtmp2.%d", d); TRY(field(h, h->vtmp2[d], nm));
    snprintf(nm, sizeof nm, "hdiv.%d", d); TRY(field(h, h->hdiv[d], nm));
    snprintf(nm, sizeof nm, "gq.%d", d); TRY(field(h, h->gq[d], nm));
    snprintf(nm, sizeof nm, "qa.%d", d); TRY(field(h, h->qa[d], nm));
  }
  TRY(field(h, h->Mc, "Mc", true)); TRY(field(h, h->Mu, "Mu", true)); TRY(field(h, h->Ml, "Ml", true));
  TRY(field(h, h->ethtot0, "ethtot0"));
  TRY(field(h, h->flx_v, "flx_v")); TRY(field(h, h->rhog_t, "rhog_t")); TRY(field(h, h->q, "q"));
  TRY(field(h, h->Qmin, "Qmin")); TRY(field(h, h->Qmax, "Qmax"));
  for (int n = 0; n < 8; ++n) { snprintf(nm, sizeof nm, "vph.%d", n); TRY(field(h, h->vph[n], nm)); }
  for (int f = 0; f < 6; ++f) {
    snprintf(nm, sizeof nm, "flx.%d", f); TRY(field(h, h->flx[f], nm));
    snprintf(nm, sizeof nm, "ch.%d", f); TRY(field(h, h->ch[f], nm));
    snprintf(nm, sizeof nm, "cm.%d", f); TRY(field(h, h->cm[f], nm));
  }
  for (int f = 0; f < 9; ++f) { snprintf(nm, sizeof nm, "xc.%d", f); TRY(field(h, h->xc[f], nm)); }
  // the pole arrays of flx/ch/cm/xc/qa are single (g,k,l[,3]) arrays: make the
  // first pole buffer of each family large enough for its (g,k,l,3) use
  {
    double* big;
    TRY(dev_alloc(h, &big, (size_t)D.npl * 3));
    h->xc[0].p = big;
    h->fields["xc.0"] = h->xc[0];
  }
  TRY(dev_alloc(h, &h->stage, (size_t)D.npt * (6 + D.nq)));
  TRY(dev_alloc(h, &h->stage_pl, (size_t)D.npl * (6 + D.nq)));
  TRY(dev_alloc(h, &h->stage_out, (size_t)D.npt * (6 + D.nq)));
  TRY(dev_alloc(h, &h->stage_out_pl, (size_t)D.npl * (6 + D.nq)));
  h->mass_blocks = (int)((D.npt2 + D.LP + 255) / 256);
  TRY(dev_alloc(h, &h->mass_part, (size_t)h->mass_blocks * 2));
  CU(cudaMalloc((void**)&h->bad, sizeof(int)));
  h->allocs.push_back(h->bad);
  CU(cudaHostAlloc((void**)&h->bad_host, sizeof(int), cudaHostAllocDefault));
  *h->bad_host = NC_BAD_NONE;
  CU(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
  {
    // the pole stream at the highest priority: its one-block kernels are
    // dispatched as soon as an SM has room instead of after the regional
    // kernel's remaining blocks, so they finish under the regional work
    int least = 0, greatest = 0;
    CU(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CU(cudaStreamCreateWithPriority(&h->stream2, cudaStreamNonBlocking, greatest));
  }
  CU(cudaEventCreateWithFlags(&h->ev_fork, cudaEventDisableTiming));
  CU(cudaEventCreateWithFlags(&h->ev_join, cudaEventDisableTiming));
  CU(cudaStreamCreateWithFlags(&h->s_h2d, cudaStreamNonBlocking));
  CU(cudaStreamCreateWithFlags(&h->s_d2h, cudaStreamNonBlocking));
  for (cudaEvent_t* e : {&h->ev_in_ready, &h->ev_in_free, &h->ev_out_ready, &h->ev_out_done, &h->ev_user})
    CU(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
  return 0;
}

int nc_create(const nc_array* arrays, int32_t narrays, nc_handle** out) {
  if (!out || !arrays || narrays <= 0) return fail(NC_ERR_ARG, "nc_create: null argument");
  *out = nullptr;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return fail(NC_ERR_CUDA, "no CUDA device");
  nc_handle* h = new nc_handle();
  int rc = create_impl(arrays, narrays, h);
  if (rc) {
    std::string keep = g_err;
    nc_destroy(h);
    g_err = keep;
    return rc;
  }
  *out = h;
  return 0;
}

void nc_destroy(nc_handle* h) {
  if (!h) return;
  if (h->gexec) cudaGraphExecDestroy(h->gexec);
  if (h->graph) cudaGraphDestroy(h->graph);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (cudaEvent_t e : h->ev_pool) cudaEventDestroy(e);
  for (void* p : h->allocs) cudaFree(p);
  if (h->bad_host) cudaFreeHost(h->bad_host);
  if (h->stream2) cudaStreamSynchronize(h->stream2);
  for (cudaStream_t st : {h->s_h2d, h->s_d2h})
    if (st) cudaStreamSynchronize(st);
  for (cudaEvent_t e : {h->ev_in_ready, h->ev_in_free, h->ev_out_ready, h->ev_out_done, h->ev_user})
    if (e) cudaEventDestroy(e);
  for (cudaStream_t st : {h->s_h2d, h->s_d2h})
    if (st) cudaStreamDestroy(st);
  if (h->ev_fork) cudaEventDestroy(h->ev_fork);
  if (h->ev_join) cudaEventDestroy(h->ev_join);
  if (h->stream2) cudaStreamDestroy(h->stream2);
  if (h->stream) cudaStreamDestroy(h->stream);
  if (g_current == h) g_current = nullptr;
  delete h;
}


int nc_upload_state(nc_handle* h, const double* prg, const double* prg_pl) {
  if (!h || !prg || !prg_pl) return fail(NC_ERR_ARG, "nc_upload_state: null argument");
  TRY(load_consts(h));
  const Dims& D = h->D;
  const int nv = 6 + D.nq;
  // copy on the upload stream once the staging buffer's last unpack is done,
  // then unpack on the library stream behind everything already queued there
  CU(cudaStreamWaitEvent(h->s_h2d, h->ev_in_free, 0));
  CU(cudaMemcpyAsync(h->stage, prg, (size_t)D.npt * nv * sizeof(double), cudaMemcpyHostToDevice, h->s_h2d));
  CU(cudaMemcpyAsync(h->stage_pl, prg_pl, (size_t)D.npl * nv * sizeof(double), cudaMemcpyHostToDevice, h->s_h2d));
  CU(cudaEventRecord(h->ev_in_ready, h->s_h2d));
  CU(cudaStreamWaitEvent(h->stream, h->ev_in_ready, 0));
  TRY(h->mixed ? unpack_state<float>(h, h->stage, h->stage_pl) : unpack_state<double>(h, h->stage, h->stage_pl));
  CU(cudaEventRecord(h->ev_in_free, h->stream));
  h->have_state = true;
  return 0;
}

// pack the state into the download staging buffer on the library stream and
// copy it out on the download stream
static int reset_bad(nc_handle* h, cudaStream_t st) {
  CU(cudaMemsetAsync(h->bad, 0x7f, sizeof(int), st));
  return 0;
}

static int download_issue(nc_handle* h, double* prg, double* prg_pl) {
  const Dims& D = h->D;
  const int nv = 6 + D.nq;
  CU(cudaStreamWaitEvent(h->stream, h->ev_out_done, 0));   // the previous download has left the buffer
  const dim3 gt((unsigned)((D.G + UI - 1) / UI), (unsigned)((D.L * nv + UC - 1) / UC), (unsigned)(D.G * D.KA));
  TRY(reset_bad(h, h->stream));
  TRY(h->mixed ? pack_state<float>(h, h->stage_out, h->stage_out_pl)
               : pack_state<double>(h, h->stage_out, h->stage_out_pl));
  CU(cudaEventRecord(h->ev_out_ready, h->stream));
  CU(cudaStreamWaitEvent(h->s_d2h, h->ev_out_ready, 0));
  CU(cudaMemcpyAsync(prg, h->stage_out, (size_t)D.npt * nv * sizeof(double), cudaMemcpyDeviceToHost, h->s_d2h));
  CU(cudaMemcpyAsync(prg_pl, h->stage_out_pl, (size_t)D.npl * nv * sizeof(double), cudaMemcpyDeviceToHost,
                     h->s_d2h));
  CU(cudaMemcpyAsync(h->bad_host, h->bad, sizeof(int), cudaMemcpyDeviceToHost, h->s_d2h));
  CU(cudaEventRecord(h->ev_out_done, h->s_d2h));
  return 0;
}

// NC_ERR_NONFINITE naming the lowest variable index the last finiteness check
// or download saw non-finite (the caller has synchronized with it)
static int bad_status(nc_handle* h, const char* what) {
  const int v = *h->bad_host;
  if (v == NC_BAD_NONE) return 0;
  return fail(NC_ERR_NONFINITE, std::string(what) + ": non-finite value in prognostic variable " + std::to_string(v) +
                                    " (0-5 RHOG..RHOGE, 6.. tracers)");
}

int nc_download_state(nc_handle* h, double* prg, double* prg_pl) {
  if (!h || !prg || !prg_pl) return fail(NC_ERR_ARG, "nc_download_state: null argument");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_download_state: no state uploaded");
  TRY(load_consts(h));
  TRY(download_issue(h, prg, prg_pl));
  CU(cudaEventSynchronize(h->ev_out_done));
  return bad_status(h, "nc_download_state");
}

int nc_check_finite(nc_handle* h) {
  if (!h) return fail(NC_ERR_ARG, "nc_check_finite: null handle");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_check_finite: no state uploaded");
  TRY(load_consts(h));
  TRY(reset_bad(h, h->stream));
  TRY(h->mixed ? finite_state<float>(h) : finite_state<double>(h));
  CU(cudaMemcpyAsync(h->bad_host, h->bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return bad_status(h, "nc_check_finite");
}

// the library stream waits for the work queued so far on the caller's stream
// (cudaStream_t; NULL is the legacy default stream)
static int after_caller(nc_handle* h, void* stream) {
  CU(cudaEventRecord(h->ev_user, (cudaStream_t)stream));
  CU(cudaStreamWaitEvent(h->stream, h->ev_user, 0));
  return 0;
}
// ... and the caller's stream waits for the library stream
static int before_caller(nc_handle* h, void* stream) {
  CU(cudaEventRecord(h->ev_user, h->stream));
  CU(cudaStreamWaitEvent((cudaStream_t)stream, h->ev_user, 0));
  return 0;
}

int nc_upload_state_device(nc_handle* h, const double* prg, const double* prg_pl, void* stream) {
  if (!h || !prg || !prg_pl) return fail(NC_ERR_ARG, "nc_upload_state_device: null argument");
  TRY(load_consts(h));
  TRY(after_caller(h, stream));
  TRY(h->mixed ? unpack_state<float>(h, prg, prg_pl) : unpack_state<double>(h, prg, prg_pl));
  TRY(before_caller(h, stream));
  h->have_state = true;
  return 0;
}

int nc_download_state_device(nc_handle* h, double* prg, double* prg_pl, void* stream) {
  if (!h || !prg || !prg_pl) return fail(NC_ERR_ARG, "nc_download_state_device: null argument");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_download_state_device: no state uploaded");
  TRY(load_consts(h));
  TRY(after_caller(h, stream));
  TRY(reset_bad(h, h->stream));
  TRY(h->mixed ? pack_state<float>(h, prg, prg_pl) : pack_state<double>(h, prg, prg_pl));
  return before_caller(h, stream);
}

int nc_download_state_async(nc_handle* h, double* prg, double* prg_pl) {
  if (!h || !prg || !prg_pl) return fail(NC_ERR_ARG, "nc_download_state_async: null argument");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_download_state_async: no state uploaded");
  TRY(load_consts(h));
  return download_issue(h, prg, prg_pl);
}

int nc_join_copies(nc_handle* h) {
  if (!h) return fail(NC_ERR_ARG, "nc_join_copies: null handle");
  CU(cudaStreamWaitEvent(h->stream, h->ev_in_ready, 0));
  CU(cudaStreamWaitEvent(h->stream, h->ev_out_done, 0));
  return 0;
}

int nc_set_block(nc_handle* h, const char* kernel, int32_t threads) {
  if (!h || !kernel) return fail(NC_ERR_ARG, "nc_set_block: null argument");
  for (int n = 0; n < TB_N; ++n) {
    if (std::strcmp(kernel, kTuneName[n]) != 0) continue;
    if (threads < 32 || threads > kTuneMax[n] || threads % 32 != 0)
      return fail(NC_ERR_ARG, std::string("nc_set_block: ") + kernel + " takes a multiple of 32 threads up to " +
                                  std::to_string(kTuneMax[n]));
    if (h->blk[n] != threads) {
      h->blk[n] = threads;
      TRY(drop_graph(h));
    }
    return 0;
  }
  return fail(NC_ERR_ARG, std::string("nc_set_block: no tunable kernel ") + kernel);
}

int nc_get_block(nc_handle* h, const char* kernel, int32_t* threads) {
  if (!h || !kernel || !threads) return fail(NC_ERR_ARG, "nc_get_block: null argument");
  for (int n = 0; n < TB_N; ++n)
    if (std::strcmp(kernel, kTuneName[n]) == 0) {
      *threads = h->blk[n];
      return 0;
    }
  return fail(NC_ERR_ARG, std::string("nc_get_block: no tunable kernel ") + kernel);
}

int nc_set_graph(nc_handle* h, int32_t enable) {
  if (!h) return fail(NC_ERR_ARG, "nc_set_graph: null handle");
  h->use_graph = enable != 0;
  return 0;
}

int nc_step(nc_handle* h, int32_t nsteps) {
  if (!h || nsteps < 0) return fail(NC_ERR_ARG, "nc_step: bad argument");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_step: no state uploaded");
  TRY(load_consts(h));
  if (!h->use_graph || h->prof) {
    h->stepped = h->stepped || nsteps > 0;
    for (int n = 0; n < nsteps; ++n) {
      if (h->prof) h->ev_used = 0;
      TRY(step_once(h));
      if (h->prof) TRY(collect_profile(h));
    }
    return 0;
  }
  if (!h->gexec) {
    long long before = h->launches;
    CU(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
    int rc = step_once(h);
    cudaGraph_t g = nullptr;
    cudaError_t ec = cudaStreamEndCapture(h->stream, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ec != cudaSuccess) return fail(NC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(ec));
    h->graph = g;
    CU(cudaGraphInstantiate(&h->gexec, h->graph, cudaGraphInstantiateFlagUseNodePriority));
    h->launches = before;
    h->graph_kernels = 0;
    {
      size_t nn = 0;
      CU(cudaGraphGetNodes(h->graph, nullptr, &nn));
      std::vector<cudaGraphNode_t> nodes(nn);
      CU(cudaGraphGetNodes(h->graph, nodes.data(), &nn));
      for (auto& node : nodes) {
        cudaGraphNodeType t;
        CU(cudaGraphNodeGetType(node, &t));
        if (t == cudaGraphNodeTypeKernel) h->graph_kernels++;
      }
    }
  }
  h->stepped = h->stepped || nsteps > 0;
  for (int n = 0; n < nsteps; ++n) {
    CU(cudaGraphLaunch(h->gexec, h->stream));
    h->launches += h->graph_kernels;
  }
  return 0;
}

int nc_run_phases(nc_handle* h, int32_t nphases) {
  if (!h || nphases < 1) return fail(NC_ERR_ARG, "nc_run_phases: bad argument");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_run_phases: no state uploaded");
  TRY(load_consts(h));
  h->stop_phase = nphases;
  int rc = step_once(h);
  h->stop_phase = 0;
  if (rc) return rc;
  CU(cudaStreamSynchronize(h->stream));
  return 0;
}

int nc_sync(nc_handle* h) {
  if (!h) return fail(NC_ERR_ARG, "nc_sync: null handle");
  CU(cudaStreamSynchronize(h->stream));
  CU(cudaStreamSynchronize(h->s_h2d));
  CU(cudaStreamSynchronize(h->s_d2h));
  return 0;
}

int nc_mass_sums(nc_handle* h, double* out, int32_t nout) {
  if (!h || !out || nout < 1) return fail(NC_ERR_ARG, "nc_mass_sums: bad argument");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_mass_sums: no state uploaded");
  TRY(load_consts(h));
  std::vector<double> part((size_t)h->mass_blocks * 2);
  for (int n = 0; n < nout && n <= h->D.nq; ++n) {
    TRY(h->mixed ? mass_sum<float>(h, n) : mass_sum<double>(h, n));
    CU(cudaMemcpyAsync(part.data(), h->mass_part, part.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CU(cudaStreamSynchronize(h->stream));
    double S = 0.0, Cc = 0.0;
    for (int b = 0; b < h->mass_blocks; ++b) {
      double x = part[b * 2];
      double t = S + x;
      if (std::fabs(S) >= std::fabs(x)) Cc += (S - t) + x;
      else Cc += (x - t) + S;
      S = t;
      Cc += part[b * 2 + 1];
    }
    out[n] = S + Cc;
  }
  return 0;
}

int nc_get_field(nc_handle* h, const char* name, double* host_reg, double* host_pl) {
  if (!h || !name) return fail(NC_ERR_ARG, "nc_get_field: null argument");
  auto it = h->fields.find(name);
  if (it == h->fields.end()) return fail(NC_ERR_ARG, std::string("unknown field ") + name);
  TRY(load_consts(h));
  const Dims& D = h->D;
  CU(cudaStreamSynchronize(h->stream));
  const bool f32 = h->field_esize[name] == (int)sizeof(float);
  if (host_reg) {
    std::vector<double> tmp((size_t)D.npt);
    if (f32) {
      std::vector<float> tf((size_t)D.npt);
      CU(cudaMemcpy(tf.data(), it->second.r, D.npt * sizeof(float), cudaMemcpyDeviceToHost));
      for (size_t n = 0; n < tf.size(); ++n) tmp[n] = tf[n];
    } else {
      CU(cudaMemcpy(tmp.data(), it->second.r, D.npt * sizeof(double), cudaMemcpyDeviceToHost));
    }
    for (int l = 0; l < D.L; ++l)
      for (int k = 0; k < D.KA; ++k)
        for (int j = 0; j < D.G; ++j)
          for (int i = 0; i < D.G; ++i)
            host_reg[(((size_t)i * D.G + j) * D.KA + k) * D.L + l] = tmp[(((size_t)l * D.KA + k) * D.G + j) * D.G + i];
  }
  if (host_pl) {
    if (f32) {
      std::vector<float> tf((size_t)D.npl);
      CU(cudaMemcpy(tf.data(), it->second.p, D.npl * sizeof(float), cudaMemcpyDeviceToHost));
      for (int n = 0; n < D.npl; ++n) host_pl[n] = tf[n];
    } else {
      CU(cudaMemcpy(host_pl, it->second.p, D.npl * sizeof(double), cudaMemcpyDeviceToHost));
    }
  }
  return 0;
}

int nc_state_pointers(nc_handle* h, int32_t v, double** reg, double** pl) {
  if (!h || v < 0 || v >= 6 + h->D.nq || !reg || !pl) return fail(NC_ERR_ARG, "nc_state_pointers: bad argument");
  TRY(f64_only(h, "nc_state_pointers"));
  FieldPair f = v < 6 ? h->P[v] : h->Pq[v - 6];
  *reg = f.r;
  *pl = f.p;
  return 0;
}

int nc_stream(nc_handle* h, void** stream) {
  if (!h || !stream) return fail(NC_ERR_ARG, "nc_stream: null argument");
  *stream = (void*)h->stream;
  return 0;
}

int nc_profile(nc_handle* h, int32_t enable) {
  if (!h) return fail(NC_ERR_ARG, "nc_profile: null handle");
  CU(cudaStreamSynchronize(h->stream));
  h->prof = enable != 0;
  h->kstats.clear();
  h->ev_used = 0;
  return 0;
}

int nc_kernel_stats(nc_handle* h, int32_t max_kernels, char* names, double* total_ms, int64_t* launches) {
  if (!h || max_kernels < 0 || (max_kernels > 0 && (!names || !total_ms || !launches)))
    return -fail(NC_ERR_ARG, "nc_kernel_stats: bad argument");
  int n = 0;
  for (const auto& kv : h->kstats) {
    if (n < max_kernels) {
      snprintf(names + (size_t)n * NC_KNAME, NC_KNAME, "%s", kv.first.c_str());
      total_ms[n] = kv.second.first;
      launches[n] = kv.second.second;
    }
    ++n;
  }
  return n;
}

// grid generation helper: spring-dynamics relaxation (see nc_grid.cuh)
static int spring_impl(int32_t L, int32_t G, double* x, double* x_pl, const unsigned char* have_sgp,
                       const int64_t* r_dst, const int64_t* r_src, int32_t nr, const int64_t* p_dst,
                       const int64_t* p_src, int32_t np, double lam, double dbar, double dt, double crit,
                       int64_t max_iter, int64_t* iters_out, std::vector<void*>& mem, cudaStream_t& st,
                       cudaGraph_t& graph, cudaGraphExec_t& gexec) {
  const size_t plane = (size_t)L * G * G;
  auto alloc = [&](void** p, size_t bytes) -> int {
    CU(cudaMalloc(p, bytes));
    mem.push_back(*p);
    return 0;
  };
  SpringDev s{};
  std::vector<double> h(plane);
  for (int b = 0; b < 2; ++b)
    for (int d = 0; d < 3; ++d) {
      TRY(alloc((void**)&s.R[b][d], plane * sizeof(double)));
      for (size_t q = 0; q < plane; ++q) h[q] = x[q * 3 + d];
      CU(cudaMemcpy(s.R[b][d], h.data(), plane * sizeof(double), cudaMemcpyHostToDevice));
    }
  for (int d = 0; d < 3; ++d) {
    TRY(alloc((void**)&s.W[d], plane * sizeof(double)));
    CU(cudaMemset(s.W[d], 0, plane * sizeof(double)));
    double pl[12];
    for (int g = 0; g < 6; ++g)
      for (int lp = 0; lp < 2; ++lp) pl[g * 2 + lp] = x_pl[(lp * 6 + g) * 3 + d];
    TRY(alloc((void**)&s.Rpl[d], sizeof(pl)));
    CU(cudaMemcpy(s.Rpl[d], pl, sizeof(pl), cudaMemcpyHostToDevice));
  }
  const void* src[4] = {r_dst, r_src, p_dst, p_src};
  const long long** dst[4] = {&s.r_dst, &s.r_src, &s.p_dst, &s.p_src};
  const int cnt[4] = {nr, nr, np, np};
  for (int n = 0; n < 4; ++n) {
    TRY(alloc((void**)dst[n], (size_t)std::max(cnt[n], 1) * sizeof(long long)));
    if (cnt[n]) CU(cudaMemcpy((void*)*dst[n], src[n], cnt[n] * sizeof(long long), cudaMemcpyHostToDevice));
  }
  TRY(alloc((void**)&s.sgp, L));
  CU(cudaMemcpy((void*)s.sgp, have_sgp, L, cudaMemcpyHostToDevice));
  TRY(alloc((void**)&s.fmax, sizeof(unsigned long long)));
  TRY(alloc((void**)&s.done, sizeof(int)));
  TRY(alloc((void**)&s.iters, sizeof(long long)));
  CU(cudaMemset(s.fmax, 0, sizeof(unsigned long long)));
  CU(cudaMemset(s.done, 0, sizeof(int)));
  CU(cudaMemset(s.iters, 0, sizeof(long long)));
  s.nr = nr; s.np = np; s.G = G; s.L = L; s.lam = lam; s.dbar = dbar; s.dt = dt; s.crit = crit;
  CU(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  const int n = G - 2;
  const unsigned bstep = (unsigned)(((long long)L * n * n + 255) / 256);
  const unsigned bcomm = (unsigned)((nr + np + 255) / 256);
  const int chunk = 256;   // even: buffer roles repeat every chunk
  CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
  for (int it = 0; it < chunk; ++it) {
    const int sb = it & 1;
    k_spring_step<<<bstep, 256, 0, st>>>(s, sb);
    k_spring_comm<<<bcomm, 256, 0, st>>>(s, 1 - sb);
    k_spring_check<<<1, 1, 0, st>>>(s);
  }
  CU(cudaStreamEndCapture(st, &graph));
  CU(cudaGraphInstantiate(&gexec, graph, 0));
  long long iters = 0;
  int done = 0;
  while (!done && iters < max_iter) {
    CU(cudaGraphLaunch(gexec, st));
    CU(cudaStreamSynchronize(st));
    CU(cudaMemcpy(&done, s.done, sizeof(int), cudaMemcpyDeviceToHost));
    CU(cudaMemcpy(&iters, s.iters, sizeof(long long), cudaMemcpyDeviceToHost));
  }
  const int fb = (int)(iters & 1);
  for (int d = 0; d < 3; ++d) {
    CU(cudaMemcpy(h.data(), s.R[fb][d], plane * sizeof(double), cudaMemcpyDeviceToHost));
    for (size_t q = 0; q < plane; ++q) x[q * 3 + d] = h[q];
    double pl[12];
    CU(cudaMemcpy(pl, s.Rpl[d], sizeof(pl), cudaMemcpyDeviceToHost));
    for (int g = 0; g < 6; ++g)
      for (int lp = 0; lp < 2; ++lp) x_pl[(lp * 6 + g) * 3 + d] = pl[g * 2 + lp];
  }
  *iters_out = iters;
  return done ? 0 : fail(NC_ERR_STATE, "spring relaxation did not converge within max_iter");
}

int nc_grid_spring(int32_t lall, int32_t gall_1d, double* x, double* x_pl, const unsigned char* have_sgp,
                   const int64_t* r_dst, const int64_t* r_src, int32_t nr, const int64_t* p_dst,
                   const int64_t* p_src, int32_t np, double lambda, double dbar, double dt, double criterion,
                   int64_t max_iter, int64_t* iterations) {
  if (!x || !x_pl || !have_sgp || !iterations || lall <= 0 || gall_1d < 4 || nr < 0 || np < 0)
    return fail(NC_ERR_ARG, "nc_grid_spring: bad argument");
  std::vector<void*> mem;
  cudaStream_t st = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  int rc = spring_impl(lall, gall_1d, x, x_pl, have_sgp, r_dst, r_src, nr, p_dst, p_src, np, lambda, dbar, dt,
                       criterion, max_iter, iterations, mem, st, graph, gexec);
  if (gexec) cudaGraphExecDestroy(gexec);
  if (graph) cudaGraphDestroy(graph);
  if (st) cudaStreamSynchronize(st);
  for (void* p : mem) cudaFree(p);
  if (st) cudaStreamDestroy(st);
  return rc;
}

// ---- restart files (fio "ADVANCED": nhm/share/mod_fio.py) ------------------
// A variable's payload in the file is the big-endian stream (region, k, ij),
// ij = j*gall_1d + i: the device field layout [l][k][j][i], byte-swapped.
static int restart_field(nc_handle* h, int32_t var, double** f) {
  if (var < 0 || var >= 6 + h->D.nq) return fail(NC_ERR_ARG, "restart: variable index out of range");
  *f = var < 6 ? h->P[var].r : h->Pq[var - 6].r;
  return 0;
}

int nc_restart_pack(nc_handle* h, int32_t var, void* host) {
  if (!h || !host) return fail(NC_ERR_ARG, "nc_restart_pack: null argument");
  TRY(f64_only(h, "nc_restart_pack"));
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_restart_pack: no state uploaded");
  double* f;
  TRY(restart_field(h, var, &f));
  TRY(load_consts(h));
  const Dims& D = h->D;
  CU(cudaStreamWaitEvent(h->stream, h->ev_out_done, 0));   // the staging buffer is free
  k_restart_swap<<<(unsigned)((D.npt + 255) / 256), 256, 0, h->stream>>>(
      (unsigned long long*)h->stage_out, (const unsigned long long*)f, (int)D.npt);
  TRY(check_launch(h, "restart_pack"));
  CU(cudaMemcpyAsync(host, h->stage_out, (size_t)D.npt * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return 0;
}

int nc_restart_unpack(nc_handle* h, int32_t var, const void* host) {
  if (!h || !host) return fail(NC_ERR_ARG, "nc_restart_unpack: null argument");
  TRY(f64_only(h, "nc_restart_unpack"));
  double* f;
  TRY(restart_field(h, var, &f));
  TRY(load_consts(h));
  const Dims& D = h->D;
  // no upload may still be using the staging buffer
  CU(cudaStreamSynchronize(h->s_h2d));
  CU(cudaStreamSynchronize(h->stream));
  CU(cudaMemcpyAsync(h->stage, host, (size_t)D.npt * sizeof(double), cudaMemcpyHostToDevice, h->stream));
  k_restart_swap<<<(unsigned)((D.npt + 255) / 256), 256, 0, h->stream>>>(
      (unsigned long long*)f, (const unsigned long long*)h->stage, (int)D.npt);
  TRY(check_launch(h, "restart_unpack"));
  if (D.KA >= 3) {
    k_restart_dummy<<<(unsigned)((D.npt2 + 255) / 256), 256, 0, h->stream>>>(f);
    TRY(check_launch(h, "restart_dummy"));
  }
  CU(cudaStreamSynchronize(h->stream));
  return 0;
}

int nc_restart_finish(nc_handle* h, const int64_t* pole_src, int32_t nsrc) {
  if (!h || (nsrc > 0 && !pole_src) || nsrc < 0 || nsrc > 64) return fail(NC_ERR_ARG, "nc_restart_finish: bad argument");
  TRY(f64_only(h, "nc_restart_finish"));
  TRY(load_consts(h));
  const Dims& D = h->D;
  PoleSrc ps{};
  ps.n = nsrc;
  for (int e = 0; e < nsrc; ++e) {
    const int64_t* r = pole_src + 5 * e;
    if (r[0] < 0 || r[0] >= 6 || r[1] < 0 || r[1] >= D.LP || r[2] < 0 || r[2] >= D.G || r[3] < 0 ||
        r[3] >= D.G || r[4] < 0 || r[4] >= D.L)
      return fail(NC_ERR_ARG, "nc_restart_finish: pole source entry out of range");
    for (int c = 0; c < 5; ++c) ps.e[e][c] = (int)r[c];
  }
  VarPtrs<double> reg{}, pol{};
  const int nv = 6 + D.nq;
  for (int v = 0; v < nv; ++v) {
    reg.v[v] = v < 6 ? h->P[v].r : h->Pq[v - 6].r;
    pol.v[v] = v < 6 ? h->P[v].p : h->Pq[v - 6].p;
  }
  if (nsrc > 0) {
    k_pole_centre<<<(unsigned)((nsrc * D.KA + 127) / 128), 128, 0, h->stream>>>(reg, pol, nv, ps);
    TRY(check_launch(h, "restart_pole_centre"));
  }
  TRY(comm_prg<double>(h));
  TRY(join_pl(h));
  CU(cudaStreamSynchronize(h->stream));
  h->have_state = true;
  return 0;
}

int nc_history_vars(nc_handle* h, const int32_t* items, int32_t nitems, int64_t nstep, double dt,
                    double* const* out) {
  if (!h || (nitems > 0 && (!items || !out)) || nitems < 0 || nitems > H_N)
    return fail(NC_ERR_ARG, "nc_history_vars: bad argument");
  TRY(f64_only(h, "nc_history_vars"));
  if (!h->hist)
    return fail(NC_ERR_STATE, "nc_history_vars: the handle was created without the HIST_* setup entries");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_history_vars: no state uploaded");
  if (!(dt > 0.0)) return fail(NC_ERR_ARG, "nc_history_vars: dt must be positive");
  bool want[H_N] = {};
  for (int n = 0; n < nitems; ++n) {
    if (items[n] < 0 || items[n] >= H_N) return fail(NC_ERR_ARG, "nc_history_vars: item id out of range");
    if (want[items[n]]) return fail(NC_ERR_ARG, "nc_history_vars: item requested twice");
    if (!out[n]) return fail(NC_ERR_ARG, "nc_history_vars: null output pointer");
    if (items[n] >= H_CL && h->hist_chem[0] < 0)
      return fail(NC_ERR_ARG, "nc_history_vars: the chemistry's columns need the HIST_chem setup entry");
    want[items[n]] = true;
  }
  TRY(load_consts(h));
  const Dims& D = h->D;
  cudaStream_t s = h->stream;
  HistArgs a;
  for (int v = 0; v < 6; ++v) a.P[v] = h->P[v].r;
  for (int v = 0; v < NC_MAXNQ; ++v) a.Pq[v] = v < D.nq ? h->Pq[v].r : nullptr;
  a.iqv = h->hist_trc[0];
  a.iql[0] = h->hist_trc[1]; a.iql[1] = h->hist_trc[2];
  a.iqs[0] = h->hist_trc[3]; a.iqs[1] = h->hist_trc[4]; a.iqs[2] = h->hist_trc[5];
  a.icl = h->hist_chem[0]; a.icl2 = h->hist_chem[1];
  a.wdiag = h->w.r;
  a.hgt = h->hist_hgt; a.coslat = h->hist_coslat; a.zsfc = h->hist_zsfc; a.IJ = h->hist_IJ;
  a.dgz = h->hist_dgz;
  a.thmean = h->hist_thmean;
  for (int n = 0; n < H_N; ++n) {
    a.out[n] = nullptr;
    if (!want[n]) continue;
    if (!h->hist_out[n]) TRY(dev_alloc(h, &h->hist_out[n], (size_t)(n < H_N3 ? D.npt : D.npt2)));
    a.out[n] = h->hist_out[n];
  }
  // interval tendencies: the previous output of each tendency field and the
  // step count of the last output that formed any (mod_history_vars.py:166-180)
  bool need_tend = false;
  for (int n = 0; n < 5; ++n) need_tend = need_tend || want[H_DU + n];
  const long long dn = (need_tend && h->hist_has_nstep) ? (long long)nstep - h->hist_nstep : 0;
  a.fac = 86400.0 / dt;
  a.fac_q = a.fac * 1.0e3;
  a.dn = (double)dn;
  for (int n = 0; n < 5; ++n) {
    a.old[n] = nullptr;
    a.tform[n] = 0;
    if (!want[H_DU + n]) continue;
    if (!h->hist_old[n]) TRY(dev_alloc(h, &h->hist_old[n], (size_t)D.npt));
    a.old[n] = h->hist_old[n];
    a.tform[n] = (h->hist_old_set[n] && dn > 0) ? 1 : 0;
  }
  const double* c = h->hist_c;
  a.LHV = c[0]; a.UNDEF = c[1]; a.PSAT0 = c[2]; a.RTEM00 = c[3]; a.CPovR_liq = c[4]; a.CPovR_ice = c[5];
  a.LovR_liq = c[6]; a.LovR_ice = c[7]; a.SAT_LL = c[8]; a.SAT_UL = c[9];
  // the state may still be arriving on the upload stream; the staging buffer
  // reused below may still be leaving on the download stream
  CU(cudaStreamWaitEvent(s, h->ev_in_ready, 0));
  CU(cudaStreamWaitEvent(s, h->ev_out_done, 0));
  if (want[H_TH_PRIME]) {
    k_history_thmean<<<(unsigned)D.KA, 256, 0, s>>>(a, h->hist_area, h->hist_thmean);
    TRY(check_launch(h, "history_thmean"));
  }
  k_history<<<(unsigned)((D.npt2 + 127) / 128), 128, 0, s>>>(a);
  TRY(check_launch(h, "history"));
  for (int n = 0; n < 5; ++n)
    if (want[H_DU + n]) h->hist_old_set[n] = true;
  if (need_tend) {
    h->hist_nstep = nstep;
    h->hist_has_nstep = true;
  }
  // each output to the host in the reference layout: (i, j, k, l) or (i, j, l)
  for (int n = 0; n < nitems; ++n) {
    const int it = items[n];
    if (it < H_N3) {
      VarPtrs<double> vp{};
      vp.v[0] = h->hist_out[it];
      const dim3 gt((unsigned)((D.G + UI - 1) / UI), (unsigned)((D.L + UC - 1) / UC), (unsigned)(D.G * D.KA));
      k_pack_t<<<gt, 256, 0, s>>>(h->stage_out, vp, 1, h->bad);   // the finiteness note is not read here
      TRY(check_launch(h, "history_pack"));
      CU(cudaMemcpyAsync(out[n], h->stage_out, (size_t)D.npt * sizeof(double), cudaMemcpyDeviceToHost, s));
    } else {
      k_pack_plane<<<(unsigned)((D.npt2 + 255) / 256), 256, 0, s>>>(h->stage_out, h->hist_out[it]);
      TRY(check_launch(h, "history_pack_plane"));
      CU(cudaMemcpyAsync(out[n], h->stage_out, (size_t)D.npt2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    }
    CU(cudaStreamSynchronize(s));
  }
  CU(cudaStreamSynchronize(s));
  return 0;
}

int nc_mass_sum_noalloc(const double* rhog, const double* rhogq, const double* gsgam2, const double* volume,
                        const double* rhog_pl, const double* rhogq_pl, const double* gsgam2_pl,
                        const double* volume_pl, int32_t gall_1d, int32_t lall, int32_t kall, int32_t kmin,
                        int32_t kmax, double* out, void* stream) {
  if (!rhog || !gsgam2 || !volume || !rhog_pl || !gsgam2_pl || !volume_pl || !out)
    return fail(NC_ERR_ARG, "nc_mass_sum_noalloc: null pointer");
  if ((rhogq == nullptr) != (rhogq_pl == nullptr))
    return fail(NC_ERR_ARG, "nc_mass_sum_noalloc: rhogq and rhogq_pl must both be given or both be null");
  if (gall_1d < 4 || lall < 1 || kall < 4 || kall > NC_MAXK || kmin < 0 || kmax < kmin || kmax >= kall)
    return fail(NC_ERR_ARG, "nc_mass_sum_noalloc: bad sizes (need gall_1d >= 4, lall >= 1, 4 <= kall <= 128, "
                            "0 <= kmin <= kmax < kall)");
  const long long cols = (long long)lall * gall_1d * gall_1d + 2;
  const long long blocks = (cols + 255) / 256;
  if (blocks > NC_NOALLOC_MASS_MAX_BLOCKS)
    return fail(NC_ERR_ARG, "nc_mass_sum_noalloc: " + std::to_string(cols) +
                                " columns exceed the fixed scratch limit of " +
                                std::to_string((long long)NC_NOALLOC_MASS_MAX_BLOCKS * 256 - 2) +
                                " (lall * gall_1d^2); use nc_mass_sums");
  double* part = nullptr;
  TRY(mass_scratch_ptr(&part));
  cudaStream_t st = (cudaStream_t)stream;
  k_mass_noalloc<<<(unsigned)blocks, 256, 0, st>>>(rhog, rhogq, gsgam2, volume, rhog_pl, rhogq_pl, gsgam2_pl,
                                                   volume_pl, gall_1d, lall, kall, kmin, kmax, part);
  CU(cudaGetLastError());
  k_mass_noalloc_fold<<<1, 1, 0, st>>>(part, (int)blocks, out);
  CU(cudaGetLastError());
  return 0;
}

int nc_divide_known(const double* x, const double* y, double* q, int64_t n, double b) {
  if (!x || !q || n < 0 || n > (int64_t)1 << 28) return fail(NC_ERR_ARG, "nc_divide_known: bad argument");
  if (!y && !(b != 0.0 && std::isfinite(b)))
    return fail(NC_ERR_ARG, "nc_divide_known: divisor must be finite and nonzero");
  if (n == 0) return 0;
  double bh = 0.0, bl = 0.0;
  if (!y) recip_pair(b, bh, bl);
  double* d = nullptr;
  const size_t bytes = (size_t)n * sizeof(double);
  CU(cudaMalloc(&d, 3 * bytes));
  cudaError_t e = cudaMemcpy(d, x, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess && y) e = cudaMemcpy(d + 2 * n, y, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_divide_known<<<(unsigned)((n + 255) / 256), 256>>>(d, y ? d + 2 * n : nullptr, d + n, (int)n, b, bh, bl);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(q, d + n, bytes, cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return fail(NC_ERR_CUDA, std::string("nc_divide_known: ") + cudaGetErrorString(e));
  return 0;
}

// ---------------------------------------------------------------------------
// tangent-linear and adjoint operators on caller device buffers (float64)
// ---------------------------------------------------------------------------
static int adj_ready(nc_handle* h, const char* what) {
  if (!h) return fail(NC_ERR_ARG, std::string(what) + ": null handle");
  TRY(f64_only(h, what));
  if (h->D.KA > NC_ADJ_K)
    return fail(NC_ERR_ARG, std::string(what) + ": kall " + std::to_string(h->D.KA) + " above the limit of " +
                                std::to_string(NC_ADJ_K) + " levels");
  if (h->D.kmin < 1 || h->D.kmax > h->D.KA - 2 || h->D.kmax <= h->D.kmin)
    return fail(NC_ERR_ARG, std::string(what) + ": needs 1 <= kmin < kmax <= kall - 2");
  return load_consts(h);
}
static unsigned col_blocks(const nc_handle* h, int pole, int tpb) {
  const long long n = pole ? 6LL * h->D.LP : h->D.npt2;
  return (unsigned)((n + tpb - 1) / tpb);
}

int nc_vsolve(nc_handle* h, int32_t pole, int32_t transpose, const double* Mc, const double* Mu, const double* Ml,
              const double* b, double* x, const double* x_fwd, double* gMc, double* gMu, double* gMl,
              void* stream) {
  TRY(adj_ready(h, "nc_vsolve"));
  if (!Mc || !Mu || !Ml || !b || !x) return fail(NC_ERR_ARG, "nc_vsolve: null pointer");
  if (x_fwd && (!transpose || !gMc || !gMu || !gMl))
    return fail(NC_ERR_ARG, "nc_vsolve: the matrix cotangents need transpose = 1 and gMc, gMu, gMl");
  TriArgs a{Mc, Mu, Ml, b, x, x_fwd, gMc, gMu, gMl, transpose ? 1 : 0};
  TRY(after_caller(h, stream));
  k_tri_solve<<<col_blocks(h, pole, 128), 128, 0, h->stream>>>(a, pole ? 1 : 0);
  TRY(check_launch(h, "vsolve"));
  return before_caller(h, stream);
}

int nc_vadv_lin(nc_handle* h, int32_t pole, int32_t mode, const double* rhogq, const double* den,
                const double* flx_v, const double* frhog, const double* in, double* out, double dt, double bcoef,
                int32_t clamp, void* stream) {
  TRY(adj_ready(h, "nc_vadv_lin"));
  if (mode < 0 || mode > 2) return fail(NC_ERR_ARG, "nc_vadv_lin: mode must be 0, 1 or 2");
  if (!rhogq || !den || !flx_v || !frhog || !out || (mode && !in)) return fail(NC_ERR_ARG, "nc_vadv_lin: null pointer");
  VadvLin a{rhogq, den, flx_v, frhog, in, out, dt, bcoef, clamp ? 1 : 0, mode};
  TRY(after_caller(h, stream));
  k_vadv_lin<<<col_blocks(h, pole, 64), 64, 0, h->stream>>>(a, pole ? 1 : 0);
  TRY(check_launch(h, "vadv_lin"));
  return before_caller(h, stream);
}

int nc_laplacian(nc_handle* h, int32_t transpose, const double* q, const double* q_pl, double* y, double* y_pl,
                 void* stream) {
  TRY(adj_ready(h, "nc_laplacian"));
  if (!q || !q_pl || !y || !y_pl) return fail(NC_ERR_ARG, "nc_laplacian: null pointer");
  if (q == y || q_pl == y_pl) return fail(NC_ERR_ARG, "nc_laplacian: input and output must not alias");
  const Dims& D = h->D;
  const long long ne = (long long)(h->nr + h->np) * D.KA;
  const unsigned gc = (unsigned)((ne + 255) / 256);
  const unsigned gr = (unsigned)((D.npt + 255) / 256), gp = (unsigned)((D.KA * D.LP + 127) / 128);
  TRY(after_caller(h, stream));
  if (!transpose) {
    if (!h->adj_work) TRY(dev_alloc(h, &h->adj_work, (size_t)D.npt + D.npl));
    double* w = h->adj_work;
    double* w_pl = h->adj_work + D.npt;
    CU(cudaMemcpyAsync(w, q, (size_t)D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaMemcpyAsync(w_pl, q_pl, (size_t)D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CommFields<double> f{};
    f.r[0] = w;
    f.p[0] = w_pl;
    f.n = 1;
    if (ne > 0) {
      k_comm<<<gc, 256, 0, h->stream>>>(f, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
      TRY(check_launch(h, "lap_comm"));
    }
    k_lap_fwd<<<gr, 256, 0, h->stream>>>(w, y);
    TRY(check_launch(h, "lap"));
    k_lap_fwd_pl<<<gp, 128, 0, h->stream>>>(w_pl, y_pl);
    TRY(check_launch(h, "lap_pl"));
  } else {
    k_lap_adj<<<gr, 256, 0, h->stream>>>(q, y);
    TRY(check_launch(h, "lap_adj"));
    k_lap_adj_pl<<<gp, 128, 0, h->stream>>>(q_pl, y_pl);
    TRY(check_launch(h, "lap_adj_pl"));
    if (ne > 0) {
      k_comm_adj_add<<<gc, 256, 0, h->stream>>>(y, y_pl, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
      TRY(check_launch(h, "comm_adj"));
      k_comm_adj_clear<<<gc, 256, 0, h->stream>>>(y, y_pl, h->r_dst, h->nr, h->p_dst, h->np);
      TRY(check_launch(h, "comm_adj_clear"));
    }
  }
  return before_caller(h, stream);
}

int nc_trc_step_lin(nc_handle* h, int32_t mode, const double* x0, const double* x0_pl, const double* in,
                    const double* in_pl, double* out, double* out_pl, void* stream) {
  TRY(adj_ready(h, "nc_trc_step_lin"));
  if (mode < 0 || mode > 2) return fail(NC_ERR_ARG, "nc_trc_step_lin: mode must be 0, 1 or 2");
  if (!x0 || !x0_pl || !out || !out_pl || (mode && (!in || !in_pl)))
    return fail(NC_ERR_ARG, "nc_trc_step_lin: null pointer");
  if (!h->stepped) return fail(NC_ERR_STATE, "nc_trc_step_lin: no step has run on this handle");
  TRY(lin_buffers(h));
  SingleStream one(h);
  TRY(after_caller(h, stream));
  if (h->prof) {   // per-kernel times of this call (nc_profile / nc_kernel_stats)
    h->ev_used = 0;
    TRY(mark(h, nullptr));
  }
  FieldPair* L = h->lin;
  TRY(trc_lin_forward(h, x0, x0_pl));
  CommFields<double> cf{};
  cf.n = 1;
  const long long ne = (long long)(h->nr + h->np) * h->D.KA;
  const unsigned gc = (unsigned)((ne + 255) / 256);
  if (mode == 0) {
    TRY(copy_out(h, out, out_pl, L[LN_X3]));
  } else if (mode == 1) {
    TRY(vadv_lin_launch(h, 1, L[LN_X0], h->P0[0], in, in_pl, L[LN_T1].r, L[LN_T1].p, false));
    TRY(hlin_tl(h));
    TRY(vadv_lin_launch(h, 1, L[LN_X2], h->rhog_t, L[LN_T2].r, L[LN_T2].p, out, out_pl, true));
  } else {
    TRY(copy_in(h, L[LN_T2], in, in_pl));
    TRY(comm_adj(h, L[LN_T2]));
    TRY(vadv_lin_launch(h, 2, L[LN_X2], h->rhog_t, L[LN_T2].r, L[LN_T2].p, L[LN_T1].r, L[LN_T1].p, true));
    TRY(hlin_ad(h));
    TRY(vadv_lin_launch(h, 2, L[LN_X0], h->P0[0], L[LN_T2].r, L[LN_T2].p, out, out_pl, false));
  }
  if (mode != 2 && ne > 0) {   // the closing exchange of PRG_var
    cf.r[0] = out;
    cf.p[0] = out_pl;
    k_comm<<<gc, 256, 0, h->stream>>>(cf, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
    TRY(check_launch(h, "lin_comm"));
  }
  if (h->prof) TRY(collect_profile(h));
  return before_caller(h, stream);
}

int nc_set_time(nc_handle* h, double time) {
  if (!h) return fail(NC_ERR_ARG, "nc_set_time: null handle");
  if (!h->trcadv) return fail(NC_ERR_STATE, "nc_set_time: the handle has no prescribed winds (trcadv)");
  TRY(load_consts(h));
  CU(cudaMemcpyAsync(h->trc_time, &time, sizeof(double), cudaMemcpyHostToDevice, h->stream));
  CU(cudaStreamSynchronize(h->stream));
  return 0;
}

int nc_trc_prepare(nc_handle* h) {
  if (!h) return fail(NC_ERR_ARG, "nc_trc_prepare: null handle");
  if (!h->trcadv) return fail(NC_ERR_STATE, "nc_trc_prepare: the handle has no prescribed winds (trcadv)");
  if (!h->have_state) return fail(NC_ERR_STATE, "nc_trc_prepare: no state uploaded");
  TRY(load_consts(h));
  const Dims& D = h->D;
  const size_t es = h->mixed ? sizeof(float) : sizeof(double);
  const cudaStream_t s = h->stream;
  // what a step of the offline advection does before its tracer advection:
  // PROG0 = PROG, PROG_mean = PROG, no density tendency
  for (int v = 0; v < 6; ++v) {
    CU(cudaMemcpyAsync(h->P0[v].r, h->P[v].r, D.npt * es, cudaMemcpyDeviceToDevice, s));
    CU(cudaMemcpyAsync(h->P0[v].p, h->P[v].p, D.npl * es, cudaMemcpyDeviceToDevice, s));
  }
  for (int v = 0; v < 5; ++v) {
    CU(cudaMemcpyAsync(h->PM[v].r, h->P[v].r, D.npt * es, cudaMemcpyDeviceToDevice, s));
    CU(cudaMemcpyAsync(h->PM[v].p, h->P[v].p, D.npl * es, cudaMemcpyDeviceToDevice, s));
  }
  CU(cudaMemsetAsync(h->frhog.r, 0, D.npt * es, s));
  CU(cudaMemsetAsync(h->frhog.p, 0, D.npl * es, s));
  h->stepped = true;
  return 0;
}

// the exchange (forward) or its adjoint on nf fields stored one after the other
static int comm_fields(nc_handle* h, double* r, double* p, int nf, bool adjoint) {
  const Dims& D = h->D;
  const long long ne = (long long)(h->nr + h->np) * D.KA;
  if (ne == 0) return 0;
  const unsigned gc = (unsigned)((ne + 255) / 256);
  for (int f = 0; f < nf; ++f) {
    double* rf = r + (size_t)f * D.npt;
    double* pf = p + (size_t)f * D.npl;
    if (!adjoint) {
      CommFields<double> cf{};
      cf.r[0] = rf;
      cf.p[0] = pf;
      cf.n = 1;
      k_comm<<<gc, 256, 0, h->stream>>>(cf, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
      TRY(check_launch(h, "op_comm"));
    } else {
      k_comm_adj_add<<<gc, 256, 0, h->stream>>>(rf, pf, h->r_dst, h->r_src, h->nr, h->p_dst, h->p_src, h->np);
      TRY(check_launch(h, "op_comm_adj"));
      k_comm_adj_clear<<<gc, 256, 0, h->stream>>>(rf, pf, h->r_dst, h->nr, h->p_dst, h->np);
      TRY(check_launch(h, "op_comm_adj_clear"));
    }
  }
  return 0;
}

int nc_exchange(nc_handle* h, int32_t transpose, double* x, double* x_pl, int32_t nf, void* stream) {
  TRY(adj_ready(h, "nc_exchange"));
  if (!x || !x_pl) return fail(NC_ERR_ARG, "nc_exchange: null pointer");
  if (nf < 1) return fail(NC_ERR_ARG, "nc_exchange: nf must be positive");
  TRY(after_caller(h, stream));
  TRY(comm_fields(h, x, x_pl, nf, transpose != 0));
  return before_caller(h, stream);
}

int nc_divergence(nc_handle* h, int32_t transpose, double* v, double* v_pl, double* y, double* y_pl, void* stream) {
  TRY(adj_ready(h, "nc_divergence"));
  if (!v || !v_pl || !y || !y_pl) return fail(NC_ERR_ARG, "nc_divergence: null pointer");
  const Dims& D = h->D;
  const unsigned gr = (unsigned)((D.npt + 255) / 256), gp = (unsigned)((D.KA * D.LP + 127) / 128);
  TRY(after_caller(h, stream));
  if (!transpose) {
    if (!h->adj_work3) TRY(dev_alloc(h, &h->adj_work3, 3 * ((size_t)D.npt + D.npl)));
    double* w = h->adj_work3;
    double* w_pl = w + 3 * (size_t)D.npt;
    CU(cudaMemcpyAsync(w, v, 3 * D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaMemcpyAsync(w_pl, v_pl, 3 * (size_t)D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    TRY(comm_fields(h, w, w_pl, 3, false));
    k_div_fwd<<<gr, 256, 0, h->stream>>>(w, y);
    TRY(check_launch(h, "div"));
    k_div_fwd_pl<<<gp, 128, 0, h->stream>>>(w_pl, y_pl);
    TRY(check_launch(h, "div_pl"));
  } else {
    k_div_adj<<<gr, 256, 0, h->stream>>>(y, v);
    TRY(check_launch(h, "div_adj"));
    k_div_adj_pl<<<gp, 128, 0, h->stream>>>(y_pl, v_pl);
    TRY(check_launch(h, "div_adj_pl"));
    TRY(comm_fields(h, v, v_pl, 3, true));
  }
  return before_caller(h, stream);
}

int nc_diffusion(nc_handle* h, int32_t transpose, const double* kh, const double* kh_pl, double* s, double* s_pl,
                 double* y, double* y_pl, void* stream) {
  TRY(adj_ready(h, "nc_diffusion"));
  if (!kh || !kh_pl || !s || !s_pl || !y || !y_pl) return fail(NC_ERR_ARG, "nc_diffusion: null pointer");
  if (s == y || s_pl == y_pl) return fail(NC_ERR_ARG, "nc_diffusion: input and output must not alias");
  const Dims& D = h->D;
  const unsigned gr = (unsigned)((D.npt + 255) / 256), gp = (unsigned)((D.KA * D.LP + 127) / 128);
  TRY(after_caller(h, stream));
  if (!transpose) {
    if (!h->adj_work) TRY(dev_alloc(h, &h->adj_work, (size_t)D.npt + D.npl));
    double* w = h->adj_work;
    double* w_pl = w + D.npt;
    CU(cudaMemcpyAsync(w, s, D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaMemcpyAsync(w_pl, s_pl, (size_t)D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    TRY(comm_fields(h, w, w_pl, 1, false));
    k_diff_fwd<<<gr, 256, 0, h->stream>>>(kh, w, y);
    TRY(check_launch(h, "diff"));
    k_diff_fwd_pl<<<gp, 128, 0, h->stream>>>(kh_pl, w_pl, y_pl);
    TRY(check_launch(h, "diff_pl"));
  } else {
    if (!h->adj_work6) TRY(dev_alloc(h, &h->adj_work6, 6 * (size_t)D.npt));
    k_diff_adj_tri<<<gr, 256, 0, h->stream>>>(kh, y, h->adj_work6);
    TRY(check_launch(h, "diff_adj_tri"));
    k_diff_adj_pt<<<gr, 256, 0, h->stream>>>(h->adj_work6, s);
    TRY(check_launch(h, "diff_adj_pt"));
    k_diff_adj_pl<<<gp, 128, 0, h->stream>>>(kh_pl, y_pl, s_pl);
    TRY(check_launch(h, "diff_adj_pl"));
    TRY(comm_fields(h, s, s_pl, 1, true));
  }
  return before_caller(h, stream);
}

int nc_diffusion_kh(nc_handle* h, double* s, double* s_pl, const double* y, const double* y_pl, double* gkh,
                    double* gkh_pl, void* stream) {
  TRY(adj_ready(h, "nc_diffusion_kh"));
  if (!s || !s_pl || !y || !y_pl || !gkh || !gkh_pl) return fail(NC_ERR_ARG, "nc_diffusion_kh: null pointer");
  const Dims& D = h->D;
  const unsigned gr = (unsigned)((D.npt + 255) / 256), gp = (unsigned)((D.KA * D.LP + 127) / 128);
  TRY(after_caller(h, stream));
  if (!h->adj_work) TRY(dev_alloc(h, &h->adj_work, (size_t)D.npt + D.npl));
  double* w = h->adj_work;
  double* w_pl = h->adj_work + D.npt;
  CU(cudaMemcpyAsync(w, s, D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  CU(cudaMemcpyAsync(w_pl, s_pl, (size_t)D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
  TRY(comm_fields(h, w, w_pl, 1, false));
  k_diff_khbar<<<gr, 256, 0, h->stream>>>(w, y, gkh);
  TRY(check_launch(h, "diff_khbar"));
  k_diff_khbar_pl<<<gp, 128, 0, h->stream>>>(w_pl, y_pl, gkh_pl);
  TRY(check_launch(h, "diff_khbar_pl"));
  return before_caller(h, stream);
}

// the 3-D (three = 1: four input components) or 2-D (three input components)
// divergence damping after the exchange of its inputs, or its adjoint
static int ddamp(nc_handle* h, int three, int32_t transpose, double* v, double* v_pl, double* y, double* y_pl,
                 void* stream, const char* name) {
  TRY(adj_ready(h, name));
  if (!v || !v_pl || !y || !y_pl) return fail(NC_ERR_ARG, std::string(name) + ": null pointer");
  if (v == y || v_pl == y_pl) return fail(NC_ERR_ARG, std::string(name) + ": input and output must not alias");
  const Dims& D = h->D;
  const int nc = three ? 4 : 3;
  const unsigned gr = (unsigned)((D.npt + 255) / 256), gp = (unsigned)((D.KA * D.LP + 127) / 128);
  TRY(after_caller(h, stream));
  if (!transpose) {
    double** wp = three ? &h->adj_work4 : &h->adj_work3;
    if (!*wp) TRY(dev_alloc(h, wp, (size_t)nc * ((size_t)D.npt + D.npl)));
    double* w = *wp;
    double* w_pl = w + (size_t)nc * D.npt;
    CU(cudaMemcpyAsync(w, v, (size_t)nc * D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaMemcpyAsync(w_pl, v_pl, (size_t)nc * D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    TRY(comm_fields(h, w, w_pl, nc, false));
    k_ddamp_fwd<<<gr, 256, 0, h->stream>>>(w, y, three);
    TRY(check_launch(h, "ddamp"));
    k_ddamp_fwd_pl<<<gp, 128, 0, h->stream>>>(w_pl, y_pl, three);
    TRY(check_launch(h, "ddamp_pl"));
  } else {
    if (!h->adj_work6) TRY(dev_alloc(h, &h->adj_work6, 6 * (size_t)D.npt));
    k_ddamp_adj_tri<<<gr, 256, 0, h->stream>>>(y, h->adj_work6, three);
    TRY(check_launch(h, "ddamp_adj_tri"));
    k_ddamp_adj_pt<<<gr, 256, 0, h->stream>>>(h->adj_work6, v, three);
    TRY(check_launch(h, "ddamp_adj_pt"));
    k_ddamp_adj_pl<<<gp, 128, 0, h->stream>>>(y_pl, v_pl, three);
    TRY(check_launch(h, "ddamp_adj_pl"));
    TRY(comm_fields(h, v, v_pl, nc, true));
  }
  return before_caller(h, stream);
}

int nc_divdamp3d(nc_handle* h, int32_t transpose, double* v, double* v_pl, double* y, double* y_pl, void* stream) {
  return ddamp(h, 1, transpose, v, v_pl, y, y_pl, stream, "nc_divdamp3d");
}

int nc_divdamp2d(nc_handle* h, int32_t transpose, double* v, double* v_pl, double* y, double* y_pl, void* stream) {
  return ddamp(h, 0, transpose, v, v_pl, y, y_pl, stream, "nc_divdamp2d");
}

int nc_gradient(nc_handle* h, int32_t transpose, double* q, double* q_pl, double* g, double* g_pl, void* stream) {
  TRY(adj_ready(h, "nc_gradient"));
  if (!q || !q_pl || !g || !g_pl) return fail(NC_ERR_ARG, "nc_gradient: null pointer");
  const Dims& D = h->D;
  const unsigned gr = (unsigned)((D.npt + 255) / 256), gp = (unsigned)((D.KA * D.LP + 127) / 128);
  TRY(after_caller(h, stream));
  if (!transpose) {
    if (!h->adj_work) TRY(dev_alloc(h, &h->adj_work, (size_t)D.npt + D.npl));
    double* w = h->adj_work;
    double* w_pl = w + D.npt;
    CU(cudaMemcpyAsync(w, q, D.npt * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CU(cudaMemcpyAsync(w_pl, q_pl, (size_t)D.npl * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    TRY(comm_fields(h, w, w_pl, 1, false));
    k_grad_fwd<<<gr, 256, 0, h->stream>>>(w, g);
    TRY(check_launch(h, "grad"));
    k_grad_fwd_pl<<<gp, 128, 0, h->stream>>>(w_pl, g_pl);
    TRY(check_launch(h, "grad_pl"));
  } else {
    k_grad_adj<<<gr, 256, 0, h->stream>>>(g, q);
    TRY(check_launch(h, "grad_adj"));
    k_grad_adj_pl<<<gp, 128, 0, h->stream>>>(g_pl, q_pl);
    TRY(check_launch(h, "grad_adj_pl"));
    TRY(comm_fields(h, q, q_pl, 1, true));
  }
  return before_caller(h, stream);
}

}  // extern "C"





