/* C ABI of the B200 NICAM-DC dynamics step (libnicamcuda.so).
 *
 * The reference drives its time step through the Python object
 * Dyn (pynicamdc/nhm/dynamics/mod_dynamics.py): dynamics_step(msc) at
 * mod_dynamics.py:1725, called once per step from pyNICAM.run
 * (pynicamdc/api.py:724), with the prognostic state in
 * prgv.PRG_var (gall_1d, gall_1d, kall, lall, 6+nq) and prgv.PRG_var_pl
 * (6, kall, 2, 6+nq) (pynicamdc/nhm/share/mod_prgvar.py:51), drained to the
 * host with Dyn.sync_prgvar_to_host (mod_dynamics.py:429).  These entry points
 * are what a "cuda" backend binds in place of that Python step: the host
 * keeps the reference's arrays and layouts; the library owns the device copy.
 *
 * Every function returns 0 on success and a non-zero status otherwise;
 * nc_last_error() returns the message.  No function aborts the process.
 * A handle is not re-entrant: one host thread drives one handle.  Several
 * handles on one device run one after another: the run constants are
 * device-global, so a call on a handle first waits for the work still queued
 * by the handle used before it.
 */
#ifndef NICAM_CUDA_H
#define NICAM_CUDA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  NC_OK = 0,
  NC_ERR_ARG = 1,      /* bad argument, missing or mis-shaped setup array */
  NC_ERR_CUDA = 2,     /* a CUDA runtime call failed */
  NC_ERR_STATE = 3,    /* call out of order (e.g. step before upload) */
  NC_ERR_NONFINITE = 4 /* non-finite value detected in the state */
};

enum { NC_F64 = 0, NC_I32 = 1, NC_I64 = 2, NC_BOOL = 3 };

/* One named host array of the setup.  Names and shapes follow the
 * reference's attributes: VMTR_* of share/mod_vmtr.py:30, OPRT_coef_* of
 * share/mod_oprt.py:65, GRD_* of share/mod_grd.py:64, GMTR_* of
 * share/mod_gmtr.py:65, bsstate rho_bs/pre_bs/tem_bs of
 * nhm/share/mod_bsstate.py:20, ppm.pntmask and adm.ADM_have_sgp, run
 * constants as 0-d arrays, and the halo plan (halo_r_dst, halo_r_src,
 * halo_p_dst, halo_p_src) composed from comm.Copy_list_* and
 * comm.Singular_list (share/mod_comm.py:1400-1561). */
typedef struct nc_array {
  const char* name;
  const void* data;
  int32_t dtype;
  int32_t ndim;
  int64_t shape[8];
} nc_array;

typedef struct nc_handle nc_handle;

/* Replaces Dyn.dynamics_setup (mod_dynamics.py:164) for the device: uploads
 * geometry, metrics and the halo plan, allocates all device work arrays.
 *
 * The optional scalar entry "precision" selects the arithmetic, as the
 * reference's Backend.configure(name, precision) does
 * (pynicamdc/share/mod_backend.py:175-185): 0 (default) float64, the
 * reference's numpy arithmetic bit for bit; 1 the mixed form: float32 work
 * fields, metrics and stencil / advection / hyperdiffusion / tracer
 * arithmetic, with the tridiagonal (HEVI) elimination and its matrix, the
 * pressure and density deviations from the reference state
 * (mod_dynamics.py:1056-1057) and the mass sums in float64.  The host state
 * and every marshal call stay float64 in both forms.  A mixed handle runs the
 * dynamics step (the offline tracer advection TRCADV included), the marshal
 * calls, nc_mass_sums, nc_check_finite and nc_get_field; nc_forcing_step,
 * nc_history_vars, the restart calls and nc_state_pointers return
 * NC_ERR_STATE for it, and the Held-Suarez and history set-up entries are
 * rejected (NC_ERR_ARG).
 *
 * Numerical filter options beyond the DIRECT hyperdiffusion (uniform
 * "Kh_coef"): the NONLINEAR1 hyperdiffusion (mod_numfilter.py:1153-1206)
 * with the entries "hdiff_nl_kh_max" (kall: the per-level upper bound,
 * (1 - height_factor) Kh_coef_maxlim + height_factor Kh_coef_minlim),
 * "hdiff_nl_minlim", "hdiff_nl_area" (AREA_ave) and "hdiff_nl_c1"
 * (2 AREA_ave^2 / dtl): Kh per cell and level from the first Laplacian
 * pass's temperature deviation, its half-level average for w; and the
 * Rayleigh sponge (mod_numfilter.py:219-271) with "rayleigh_coef" and
 * "rayleigh_coef_h" (kall: alpha_r times the height factor on full and
 * half levels) and optionally "rayleigh_only_w". */
int nc_create(const nc_array* arrays, int32_t narrays, nc_handle** out);

/* Marshal-in of the prognostic state (mod_dynamics.py:1876-1880) from host
 * memory in the reference layout: prg (gall_1d, gall_1d, kall, lall, 6+nq),
 * prg_pl (6, kall, 2, 6+nq), both C-order float64.  The copy runs on the
 * handle's upload stream and the steps queued after this call wait for it;
 * from pinned host memory it is asynchronous (keep the host buffer unchanged
 * until nc_sync), from pageable memory the call returns after the copy. */
int nc_upload_state(nc_handle* h, const double* prg, const double* prg_pl);

/* Marshal-out (Dyn.sync_prgvar_to_host, mod_dynamics.py:429-440) into host
 * memory in the same layout, after every step queued before the call;
 * returns when the host arrays hold the state.  The copy also checks every
 * value: if the state holds a NaN or infinity the arrays are still filled and
 * the call returns NC_ERR_NONFINITE, naming the lowest such variable index
 * (the reference has no such check; its nearest is the opt-in device checksum
 * of pynicamdc/api.py:878-900). */
int nc_download_state(nc_handle* h, double* prg, double* prg_pl);

/* Device-memory marshal for a PyTorch (or any CUDA) host: the same layouts as
 * nc_upload_state / nc_download_state, but prg and prg_pl are device pointers
 * (e.g. torch.float64 CUDA tensors of shapes (gall_1d, gall_1d, kall, lall,
 * 6+nq) and (6, kall, 2, 6+nq), contiguous), and the work is ordered against
 * the caller's `stream` (a cudaStream_t; NULL for the legacy default stream):
 * it starts after what is queued on `stream` and what is queued on `stream`
 * afterwards follows it.  Replaces the host drain of Dyn.sync_prgvar_to_host
 * (mod_dynamics.py:429-440) and the marshal-in of mod_dynamics.py:1876-1880
 * when the state lives in device tensors.  No finiteness status (use
 * nc_check_finite). */
int nc_upload_state_device(nc_handle* h, const double* prg, const double* prg_pl, void* stream);
int nc_download_state_device(nc_handle* h, double* prg, double* prg_pl, void* stream);

/* Finiteness of the device state (every prognostic and tracer, halo and
 * ghost levels included): 0, or NC_ERR_NONFINITE naming the lowest variable
 * index that holds a NaN or infinity.  Waits for the steps queued before it.
 * The reference's counterpart is its opt-in device checksum
 * (pynicamdc/api.py:878-900, PYNICAM_DEV_CHECKSUM). */
int nc_check_finite(nc_handle* h);

/* nc_download_state without the wait: the copy runs on the handle's download
 * stream, overlapping the steps queued after this call (into pinned host
 * memory); the host arrays hold the state after nc_sync.  No counterpart in
 * the reference (its drain to host is synchronous). */
int nc_download_state_async(nc_handle* h, double* prg, double* prg_pl);

/* Make the handle's stream wait for the last upload and download copies, so
 * that work or an event queued on it afterwards follows them. */
int nc_join_copies(nc_handle* h);

/* nsteps large steps of Dyn.dynamics_step (mod_dynamics.py:1725-2741) on the
 * device-resident state.  Asynchronous on the handle's stream. */
int nc_step(nc_handle* h, int32_t nsteps);

/* Capture one large step as a CUDA graph and replay it (default on). */
int nc_set_graph(nc_handle* h, int32_t enable);

/* Threads per block of one column / point kernel of the step, named as in
 * nc_kernel_stats: "diag", "vi_solve", "vi_energy", "vp0_c", "gtend",
 * "hdiff1", "post", "split_init", "trc_vflux", "trc_vadv", "trc_remap",
 * "trc_qout", "trc_apply", "trc_rhog".  A multiple of 32 up to the kernel's
 * launch bound (128 for diag, vi_solve and vi_energy, 256 for vp0_c, 1024 for
 * the others); the default is 128 (256 for vp0_c).  Changing it drops the
 * captured step graph.  The knobs of the project's autotuner
 * (pynicam-dc_b200/autotune.py); no counterpart in the reference, whose
 * jax backend leaves launch shapes to XLA. */
int nc_set_block(nc_handle* h, const char* kernel, int32_t threads);
int nc_get_block(nc_handle* h, const char* kernel, int32_t* threads);


/* Wait for the handle's streams (steps, uploads and downloads). */
int nc_sync(nc_handle* h);

/* Global sums of the embudget monitor (nhm/share/mod_embudget.py:74-80,
 * _gsum = sum of var * VMTR_VOLUME over the interior): out[0] total air mass
 * sum(rho*VOLUME), out[1 + n] tracer n mass sum(rho*q_n*VOLUME), n < nq.
 * Float64 with compensated (Neumaier) summation on the device. */
int nc_mass_sums(nc_handle* h, double* out, int32_t nout);


/* Device pointers of the resident state, for callers that keep the state in
 * their own device memory pipeline: field v (0..5 PROG, 6.. tracers) regional
 * [l][k][j][i] and pole (g,k,l).  Pointers stay valid until nc_destroy. */
int nc_state_pointers(nc_handle* h, int32_t v, double** reg, double** pl);

/* Number of kernels the library launched since the handle was created. */
int64_t nc_kernel_launches(nc_handle* h);

/* The CUDA stream (cudaStream_t) every call of this handle is ordered on, for
 * callers that time or order their own work against it. */
int nc_stream(nc_handle* h, void** stream);

/* Per-kernel device timing (measurement aid, no counterpart in the reference):
 * while enabled, nc_step launches eagerly and records an event after every
 * kernel; a kernel's time is the gap to the preceding event on the stream.
 * Enabling or disabling clears the totals. */
int nc_profile(nc_handle* h, int32_t enable);

/* Totals of the profiled steps: up to max_kernels entries of kernel name
 * (48-byte slots in names), summed milliseconds and launch count.  Returns the
 * number of distinct kernels (which may exceed max_kernels), or a negative
 * status on a bad argument. */
int nc_kernel_stats(nc_handle* h, int32_t max_kernels, char* names, double* total_ms, int64_t* launches);

/* Grid generation helper (no counterpart in the reference's step interface;
 * restates the spring-dynamics smoothing of prep/hgrid/mod_mkgrd.py:204-320).
 * x (lall, gall_1d, gall_1d, 3) region-major unit vectors with halos filled,
 * x_pl (2, 6, 3) pole points, both updated in place; the halo plan arrays are
 * those of nc_create (halo_r_dst, halo_r_src, halo_p_dst, halo_p_src).  Runs
 * until max |F|/lambda < criterion (NC_ERR_STATE after max_iter iterations);
 * the iteration count is written to *iterations.  Synchronous; allocates and
 * frees its own device memory. */
int nc_grid_spring(int32_t lall, int32_t gall_1d, double* x, double* x_pl, const unsigned char* have_sgp,
                   const int64_t* r_dst, const int64_t* r_src, int32_t nr, const int64_t* p_dst,
                   const int64_t* p_src, int32_t np, double lambda, double dbar, double dt, double criterion,
                   int64_t max_iter, int64_t* iterations);

/* Allocation-free air or tracer mass sum.  No counterpart in the reference.
 * For callers that may not call cudaMalloc: code that runs inside another
 * framework's memory manager (a caching allocator that owns the device memory,
 * an XLA/JAX custom call), where a new allocation either fails or is
 * forbidden.  Creating
 * a handle (nc_create) allocates, so this entry point takes no handle: the
 * caller passes its own device arrays in the library's device layout --
 * regional (lall, kall, gall_1d, gall_1d) C-order, pole (6, kall, 2) -- and a
 * device output of one double, and the call is ordered on `stream` (a
 * cudaStream_t; NULL for the legacy default stream).  out[0] = sum over
 * interior cells and the two pole points, levels kmin..kmax, of
 * num / gsgam2 * volume with num = rhogq if given, else rhog: the same
 * compensated sum, in the same order, as nc_mass_sums.
 * kall must be the leading level extent of the caller's arrays (4..128).
 * Limit: lall * gall_1d^2 + 2 <= 1,048,576 columns (grid level 8 at rlevel 1
 * uses 676,002); larger grids get NC_ERR_ARG.  The block partial sums live in
 * one fixed 64 KiB device array that every GPU loading the library keeps
 * until the process exits; every call overwrites the slots it reads, so no
 * state needs clearing between calls, but calls that run concurrently on the
 * GPU (different streams, overlapping) race on it and must be serialized by
 * the caller.  The first call on each device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current and keeps it for
 * the life of the process (the device's primary context must not be reset
 * meanwhile); make that first call before any stream capture.  Asynchronous:
 * read out after the stream is synchronized. */
int nc_mass_sum_noalloc(const double* rhog, const double* rhogq, const double* gsgam2, const double* volume,
                        const double* rhog_pl, const double* rhogq_pl, const double* gsgam2_pl,
                        const double* volume_pl, int32_t gall_1d, int32_t lall, int32_t kall, int32_t kmin,
                        int32_t kmax, double* out, void* stream);

/* Dyn.forcing_step (pynicamdc/nhm/dynamics/mod_dynamics.py:597-735) for
 * AF_TYPE 'HELD-SUAREZ' (nhm/forcing/mod_af_heldsuarez.py, dry case, applied as
 * in nhm/forcing/mod_forcing.py:14-28 / :323-349): diagnostics of the current
 * prognostic, Rayleigh friction and Newtonian temperature relaxation applied
 * to RHOGV{X,Y,Z} and RHOGE over kmin..kmax with the large time step, then
 * the halo exchange of PRG_var.  The poles are not forced, as in the
 * reference's host path.  Needs the handle to have been created with the
 * setup entries "AF_hs_lat_terms" ((gall_1d, gall_1d, 1, lall, 3): |sin lat|^2,
 * |cos lat|^2, |cos lat|^4 of GRD_LAT[:, :, K0, :]) and "PRE00"; otherwise
 * NC_ERR_STATE.  Asynchronous on the handle's stream, like nc_step.
 *
 * For AF_TYPE 'DCMIP' with Kessler warm-rain microphysics only (forcing_dcmip
 * USE_Kessler, the scheme set of DCMIP2016 case 1-3; nhm/forcing/
 * mod_forcing.py:207-321, mod_af_dcmip.py:129-230, kessler.py): the handle is
 * created with "AF_dcmip_kessler_zf" (GRD_vz[..., GRD_Z], (gall_1d, gall_1d,
 * kall, lall)), "PRE00", RAIN_TYPE WARM ("NQW_END" = 2: vapour, cloud, rain; the
 * simple physics alone also runs with RAIN_TYPE DRY, "NQW_END" = 0)
 * and optionally "AF_negative_fixer" / "AF_update_tot_dens" (the reference's
 * forcing_param, defaults 0 / 1).  Every regional column: diagnostics, dry
 * mixing ratios, the microphysics with its sedimentation sub-cycles, the
 * water and energy tendencies applied to the tracers, RHOGE and (with
 * update_tot_dens) RHOG, then the exchange.  exp and pow are CUDA's, so
 * results can differ from numpy's in the last bits.  The precipitation rate
 * of the step per column is read with nc_forcing_precip.  With the DCMIP
 * terminator toy chemistry as well (USE_ToyChemistry, CHEM_TYPE PASSIVE;
 * mod_af_dcmip.py:171-187, terminator.py:20-70), the handle is also created
 * with "AF_dcmip_chem" (int64 [NCHEM_STR, NCHEM_END], the Cl and Cl2 tracer
 * indices, both outside the water range) and "AF_dcmip_lat" / "AF_dcmip_lon"
 * (GRD_LAT / GRD_LON[:, :, K0, :] in radians, (gall_1d, gall_1d, 1, lall));
 * the Cl / Cl2 tendencies (per dry air, analytic over dt; sin, cos, exp and
 * sqrt are CUDA's) join the tracer tendencies on kmin..kmax.  The optional
 * "AF_dcmip_schemes" (int64 [Kessler, simple physics, large-scale
 * condensation(, moist Held-Suarez(, Bryan boundary layer))], default
 * [1, 0, 0]) adds the DCMIP simple physics (USE_SimpleMicrophys,
 * nhm/forcing/simple_physics.py with the RJ2012 boundary layer, or the Bryan
 * one, SM_PBL_Bryan; mod_af_dcmip.py:230-317) or runs it alone: its surface
 * fluxes, implicit boundary-layer diffusion of u, v, potential temperature
 * and vapour, and optional large-scale condensation, from the same state as
 * Kessler, with momentum, vapour and energy tendencies and precipitation
 * added to Kessler's.  It reads "AF_dcmip_zh" (GRD_vz[..., GRD_ZH], (gall_1d,
 * gall_1d, kall, lall)), "AF_dcmip_zsfc" (GRD_zs at K0), "AF_dcmip_tsurf" (the
 * sea-surface temperature per column) and "AF_dcmip_ij" (GMTR_p IX, IY, IZ,
 * JX, JY, JZ at K0), all (gall_1d, gall_1d, 1, lall[, 6]).  The fourth
 * switch (DCMIP2016 case 2-1, moist Held-Suarez) applies the Held-Suarez
 * relaxation with the moist equilibrium profile (T_eq0 294 K, DT_y 65 K) on
 * top: its momentum tendency replaces the others', its energy tendency adds
 * (mod_forcing.py:278-287); it reads "AF_dcmip_hs_lat_terms" (as
 * "AF_hs_lat_terms"), and the simple physics then takes the Held-Suarez
 * sea-surface temperature and four times the exchange coefficient. */
int nc_forcing_step(nc_handle* h);

/* The precipitation rate [m/s] of the last DCMIP Kessler forcing step per
 * column, into host memory (gall_1d, gall_1d, lall) (the reference's
 * frc.precip); synchronous.  NC_ERR_STATE without Kessler forcing. */
int nc_forcing_precip(nc_handle* h, double* host);

/* Restart files in the reference's fio format (input/output_io_mode
 * "ADVANCED", nhm/share/mod_fio.py), read and written from the device state:
 * every variable is stored as a big-endian float64 stream (region, k, ij) with
 * ij = j*gall_1d + i, which is the device field layout byte-swapped, so the
 * payloads move without a host transposition; the headers are the caller's.
 * var: 0..5 RHOG, RHOGVX, RHOGVY, RHOGVZ, RHOGW, RHOGE; 6.. the tracers.
 *
 * nc_restart_pack: writes the regional payload of `var` (lall*kall*gall_1d^2
 * doubles, file byte order) into `host` (Prgvar.restart_output,
 * nhm/share/mod_prgvar.py:182-216, prognostic items).  Synchronous.
 *
 * nc_restart_unpack: loads the regional field `var` from such a payload,
 * repairing non-finite values on the dummy levels as fio_read does
 * (mod_fio.py:73-84).  Synchronous.
 *
 * nc_restart_finish: after every variable is loaded, COMM_var
 * (share/mod_comm.py:2172-2300): each pole centre takes the value of its
 * source cell (pole_src: nsrc rows of int64 [pole g, pole l, i, j, l], the
 * p2r copies whose regional side is the region the pole belongs to), then the
 * halo exchange of the whole state.  The state is then the handle's
 * (Prgvar._read_prognostic_restart, mod_prgvar.py:266-306).  nsrc <= 64. */
int nc_restart_pack(nc_handle* h, int32_t var, void* host);
int nc_restart_unpack(nc_handle* h, int32_t var, const void* host);
int nc_restart_finish(nc_handle* h, const int64_t* pole_src, int32_t nsrc);

/* Dyn.history_vars_step (pynicamdc/nhm/dynamics/mod_dynamics.py:737-772 ->
 * Hvar.history_vars, pynicamdc/nhm/driver/mod_history_vars.py:30-186) on the
 * state the handle holds: the derived history diagnostics, computed on the
 * device and copied to host arrays in the reference's layout.  items[n] (n <
 * nitems) are item ids, written to out[n]:
 *   0 ml_u, 1 ml_v, 2 ml_w, 3 ml_th, 4 ml_thv, 5 ml_omg, 6 ml_pres, 7 ml_tem,
 *   8 ml_rho, 9 ml_hgt, 10 ml_mse, 11 ml_rh, 12 ml_rha, 13 ml_rhi, 14 ml_du,
 *   15 ml_dv, 16 ml_dw, 17 ml_dtem, 18 ml_dq, 19 ml_ucos, 20 ml_vcos,
 *   21 ml_th_prime                      -> (gall_1d, gall_1d, kall, lall)
 *   22 sl_ps, 23 sl_pw, 24 sl_lwp, 25 sl_iwp, 26 sl_u850, 27 sl_v850,
 *   28 sl_w850, 29 sl_t850, then ids 30-41 the same four at 500, 250 and
 *   100 hPa, 42 sl_cl, 43 sl_cl2, 44 sl_cly (the terminator chemistry's
 *   column means; AF_TYPE 'DCMIP' only)   -> (gall_1d, gall_1d, lall)
 * (the reference's I/O order, share/mod_io.py:251-261).  The tendencies ml_d*
 * are stateful as in the reference: the first output of each is zero, later
 * ones (previous - current) * 86400 / dt / (nstep - nstep of the last output
 * that formed tendencies), dq in g/kg/day; nstep is the model step count
 * (TIME_cstep), dt the large time step.  The half-level w at the boundary rows
 * is the one the last nc_step left (zero before the first step).  Needs the
 * setup entries HIST_hgt (GRD_vz Z, (gall_1d, gall_1d, kall, lall)),
 * HIST_coslat, HIST_zsfc, HIST_area (cos GRD_LAT, GRD_zs ZSFC, GMTR_area at K0;
 * (gall_1d, gall_1d, 1, lall)), HIST_IJ (GMTR_p IX, IY, IZ, JX, JY, JZ at K0;
 * (gall_1d, gall_1d, 1, lall, 6)), HIST_dgz (kall), HIST_consts (LHV, UNDEF,
 * PSAT0, RTEM00, CPovR_liq, CPovR_ice, LovR_liq, LovR_ice, SATURATION_LLIMIT_TEMP,
 * SATURATION_ULIMIT_TEMP) and HIST_tracers (int64 I_QV, I_QC, I_QR, I_QI, I_QS,
 * I_QG, -1 where absent), with PRE00; otherwise NC_ERR_STATE.  Ids 42-44 also
 * need HIST_chem (int64 NCHEM_STR, NCHEM_END), else NC_ERR_ARG.  Synchronous. */
int nc_history_vars(nc_handle* h, const int32_t* items, int32_t nitems, int64_t nstep, double dt,
                    double* const* out);


/* Tangent-linear and adjoint operators of the step, for differentiation
 * (the reference differentiates its jax backend with jax.vjp; these are the
 * hand-written counterparts of the operators named below).  They work on
 * caller device buffers in the handle's device layout -- regional fields
 * [l][k][j][i] of lall*kall*gall_1d^2 doubles, pole fields [g][k][lp] of
 * 6*kall*2 doubles -- take the run constants, geometry and halo plan from
 * the handle, are ordered after the work queued on the caller's `stream`
 * (cudaStream_t, NULL the legacy default stream) and before what the caller
 * queues there next.  Float64 handles with kall <= 64 only (NC_ERR_STATE for
 * a mixed handle, NC_ERR_ARG above 64 levels).
 *
 * nc_vsolve: the HEVI vertical implicit system of kernels/virhowsolver.py:
 * 67-122 per column (pole = 0: the regional columns, buffers regional;
 * pole = 1: the pole columns, buffers pole): rows n = kmin+1..kmax of
 * Ml[n] x[n-1] + Mc[n] x[n] + Mu[n] x[n+1] = b[n] solved by the Thomas
 * algorithm, x zero on the other levels.  transpose = 1 solves with the
 * transposed matrix (the adjoint: b is the cotangent of x, x receives the
 * cotangent of b); with x_fwd (the forward solution) it also writes the
 * matrix cotangents gMc[n] = -x[n] x_fwd[n], gMu[n] = -x[n] x_fwd[n+1],
 * gMl[n] = -x[n] x_fwd[n-1] (zero outside the system).
 *
 * nc_vadv_lin: one vertical tracer advection step with the vertical Thuburn
 * limiter (mod_src_tracer.py:389-533 and 1909-2074) at the tracer mass
 * rhogq, for fixed density den, vertical mass flux flx_v, density tendency
 * frhog (the limiter's d = bcoef * frhog / den * dt) and the clamp of tiny
 * negatives (clamp != 0).  mode 0 writes the step's result F(rhogq) to out;
 * mode 1 the tangent-linear dF(in); mode 2 the adjoint dF^T(in).  The
 * limiter's branches are those taken at rhogq (the active-branch
 * linearisation).  The halo and ghost levels of out are zero in modes 0/1.
 *
 * nc_laplacian: y = L(C(q)), the halo exchange C of the handle's plan
 * followed by the hexagonal Laplacian of kernels/oprtlaplacian.py:41-70 on
 * the interior cells and the pole points (other cells of y zero);
 * transpose = 1 writes y = C^T L^T q, the adjoint, with the exchange's
 * adjoint adding each halo value into its source cell (atomically: the
 * order of those additions, and so the last bits, may vary between calls).
 * q and y must not alias.  The forward form allocates one scratch copy of
 * a field in the handle on its first call. */
int nc_vsolve(nc_handle* h, int32_t pole, int32_t transpose, const double* Mc, const double* Mu, const double* Ml,
              const double* b, double* x, const double* x_fwd, double* gMc, double* gMu, double* gMl,
              void* stream);
int nc_vadv_lin(nc_handle* h, int32_t pole, int32_t mode, const double* rhogq, const double* den,
                const double* flx_v, const double* frhog, const double* in, double* out, double dt, double bcoef,
                int32_t clamp, void* stream);
int nc_laplacian(nc_handle* h, int32_t transpose, const double* q, const double* q_pl, double* y, double* y_pl,
                 void* stream);

/* nc_divergence: y = D(C(v)), the halo exchange of the three components
 * then the divergence of kernels/fluxconv.py:52-108 (OPRT_divergence) on the
 * interior cells and the pole points (other cells of y zero); v holds the
 * three components one after the other (3 x lall*kall*gall_1d^2 regional,
 * 3 x 6*kall*2 pole values).  transpose = 1 reads y and writes v = C^T D^T y.
 * nc_gradient: g = Grad(C(q)) (kernels/oprtgradient.py:45-88,
 * OPRT_gradient), g the three components one after the other; transpose = 1
 * reads g and writes q = C^T Grad^T g.  The buffer written must not alias the
 * one read.  The forward forms allocate a scratch copy in the handle on their
 * first call; the adjoints add with atomics (last bits may vary). */
int nc_divergence(nc_handle* h, int32_t transpose, double* v, double* v_pl, double* y, double* y_pl, void* stream);
int nc_gradient(nc_handle* h, int32_t transpose, double* q, double* q_pl, double* g, double* g_pl, void* stream);

/* The Kh-weighted horizontal diffusion of the hyperdiffusion's scalar pass
 * (kernels/oprtdiffusion.py, OPRT_diffusion; mod_numfilter.py:1219-1240)
 * after the halo exchange, and its adjoint, float64, on device buffers in the
 * library's field layout ordered on the caller's stream: y = Dk(C(s)) on
 * interior cells and the pole point (other cells zero) for the coefficient
 * field kh (rhog x CVdry x Kh or rhog x hdiff_fact_rho x Kh in the step; given
 * for every point and pole point, held fixed); transpose = 1 reads y and
 * writes s = C^T Dk^T y.  The buffer written must not alias the one read; the
 * forward allocates a scratch copy in the handle on its first call, the
 * adjoint a six-field scratch and adds with atomics in its exchange. */
int nc_diffusion(nc_handle* h, int32_t transpose, const double* kh, const double* kh_pl, double* s, double* s_pl,
                 double* y, double* y_pl, void* stream);

/* The Kh-weighted diffusion's coefficient cotangent: gkh = the derivative of
 * <y, Dk(C(s))> with respect to kh (the diffusion is bilinear in s and kh;
 * kernels/oprtdiffusion.py), every regional point and pole row written, s
 * exchanged in a scratch copy; float64 device buffers, caller's stream. */
int nc_diffusion_kh(nc_handle* h, double* s, double* s_pl, const double* y, const double* y_pl, double* gkh,
                    double* gkh_pl, void* stream);

/* The halo exchange (share/mod_comm.py:1563-1644: region edges, pole rows,
 * singular points) of nf float64 fields in place, device buffers in the
 * library's field layout, fields one after the other, ordered on the
 * caller's stream; transpose = 1 applies its adjoint in place (each halo
 * value added into its source, the halo values then zeroed). */
int nc_exchange(nc_handle* h, int32_t transpose, double* x, double* x_pl, int32_t nf, void* stream);

/* The divergence damping's two operators (mod_numfilter.py:2032-2268) after
 * the halo exchange of their inputs, and their adjoints, float64, device
 * buffers in the library's field layout, components one after the other,
 * ordered on the caller's stream.  nc_divdamp3d: y = D3(C(v)), v the four
 * momenta (rhogvx, rhogvy, rhogvz, rhogw), y three components on interior
 * cells and the pole point, levels kmin..kmax (kernels/oprt3ddivdamp.py:
 * 50-237, the singular-point fix included).  nc_divdamp2d: y = D2(C(v)), v
 * and y three components, every level (kernels/oprtdivdamp.py:54-173).
 * transpose = 1 reads y and writes v = C^T D^T y.  The buffer written must
 * not alias the one read; the forward forms allocate a scratch copy in the
 * handle on their first call, the adjoints a scratch of six fields and add
 * with atomics in the exchange's adjoint. */
int nc_divdamp3d(nc_handle* h, int32_t transpose, double* v, double* v_pl, double* y, double* y_pl, void* stream);
int nc_divdamp2d(nc_handle* h, int32_t transpose, double* v, double* v_pl, double* y, double* y_pl, void* stream);

/* nc_trc_step_lin: the tracer advection of one step (mod_src_tracer.py:
 * 83-1228 as the step runs it: vertical step, horizontal step with the
 * MIURA2004 face values and the horizontal Thuburn limiter of 2190-2605,
 * the density update, vertical step with the clamp, then the closing halo
 * exchange of PRG_var, mod_dynamics.py:2726) for one tracer mass x0 with the
 * winds, densities and density tendency of the last step this handle ran
 * (PROG_mean, PROG at the step's start and frhog as that step left them;
 * NC_ERR_STATE if no step has run).  mode 0 writes the step's tracer mass
 * T(x0) -- equal, bit for bit, to what the step made of that tracer; mode 1
 * the tangent-linear dT(x0) in; mode 2 the adjoint dT(x0)^T in.  Every min /
 * max of both limiters is linearised on the branch the forward takes at x0
 * (the active-branch linearisation).  Device-layout buffers as above
 * (regional x0, in, out; pole x0_pl, in_pl, out_pl).  The forward stages are
 * recomputed in every call (they are not kept between calls); the first call
 * allocates sixteen float64 work fields in the handle.  The adjoint
 * accumulates with atomic additions, so its last bits may vary between
 * calls. */
int nc_trc_step_lin(nc_handle* h, int32_t mode, const double* x0, const double* x0_pl, const double* in,
                    const double* in_pl, double* out, double* out_pl, void* stream);

/* The model time of an offline-advection handle's prescribed winds
 * (setup entry "trcadv": 1 for the DCMIP 1-1 deformational flow, 2 for the
 * DCMIP 1-2 Hadley-like circulation, mod_af_trcadv.py:22-149; the time
 * starts at 0 and every step adds dtl).  Re-running
 * steps from stored states (as the tracer-transport adjoint does) needs the
 * time of each state set back.  NC_ERR_STATE for a handle without
 * prescribed winds; synchronous. */
int nc_set_time(nc_handle* h, double time);

/* For an offline-advection handle: puts the winds of the uploaded state on
 * the handle as its step's tracer advection reads them (PROG_mean = PROG,
 * PROG at the step's start = PROG, no density tendency; mod_dynamics.py:
 * 2030-2085) without running the step, so that nc_trc_step_lin linearises
 * the step from that state.  NC_ERR_STATE without prescribed winds or
 * without a state. */
int nc_trc_prepare(nc_handle* h);

const char* nc_last_error(void);

void nc_destroy(nc_handle* h);

#ifdef __cplusplus
}
#endif

/* Test and debugging hooks (nc_run_phases, nc_get_field, nc_divide_known)
 * are declared in nicam_cuda_debug.h. */

#endif /* NICAM_CUDA_H */
