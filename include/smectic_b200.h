/*
 * smectic_b200.h -- C-ABI of the B200-native smectic3D time loop.
 *
 * The reference (evitral/smectic3D) has no library boundary: each program
 * integrates the Swift-Hohenberg model inside one main().  This header is the
 * boundary that replaces exactly that loop body and its diagnostics while
 * keeping main()'s inputs (the compile-time constants, the initial condition)
 * and outputs (psi in the reference's array layouts, L1, energy, surface
 * files).  Every entry point returns an int status (SH_OK = 0); no exception or
 * CUDA type crosses the boundary.  One handle owns its device memory and its
 * CUDA stream; use one handle per host thread.
 */
#ifndef SMECTIC_B200_H
#define SMECTIC_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define SH_OK 0
#define SH_EINVAL 1        /* bad argument or parameter combination            */
#define SH_ENOMEM 2        /* device or pinned host allocation failed          */
#define SH_ENONFINITE 3    /* the state became NaN/Inf                          */
#define SH_ETIMEOUT 4      /* a bounded device wait gave up                     */
#define SH_ECUDA 5         /* a CUDA call failed (message in sh_last_error)     */
#define SH_EUNSUPPORTED 6  /* size / option not built into this library        */
#define SH_ESTATE 7        /* call out of order (e.g. step before set_psi)      */

/* boundary (transform family) */
#define SH_PERIODIC 0      /* R2C / C2R  (periodicFFT/pf3d.cpp:226-291)           */
#define SH_NEUMANN 1       /* REDFT10 / REDFT01 (cosFFT/mesabi/cosNoAdvMorph.cpp:249-262) */
/* nonlinearity */
#define SH_QUINTIC 0       /* beta psi^3 - gamma psi^5 (periodicFFT/pf3d.cpp:368-369) */
#define SH_QUAD_CUBIC 1    /* beta psi^2 - gamma psi^3                           */
/* time scheme */
#define SH_CNAB2 0         /* Crank-Nicolson + Adams-Bashforth 2 (periodicFFT/pf3d.cpp:476-478) */
#define SH_IMEX_EULER 1    /* (psihat + dt Nhat) / (1 - dt L)                     */
/* arithmetic of fields and transforms */
#define SH_FP64 0
#define SH_FP32 1
#define SH_FP32_UPDATE64 2 /* FP32 fields and transforms; the plain step's CNAB2 multipliers
                              and update in FP64, which keeps long runs within 1e-6 of FP64 */
/* gradient and mixed derivatives of the Neumann curvature pass */
#define SH_CURV_DIFFERENCE 0 /* centred differences, one-sided at the walls (cosNoAdvMorphCurv.cpp:811-940) */
#define SH_CURV_SPECTRAL 1   /* exact derivatives of the cosine series (sine series through the cosine pair) */
/* host array layouts of psi */
#define SH_LAYOUT_DENSE 0  /* (i*N + j)*N + k       (cosFFT/mesabi/cosNoAdvMorph.cpp:296) */
#define SH_LAYOUT_PADDED 1 /* (i*N + j)*2(N/2+1) + k (periodicFFT/pf3d.cpp:312)         */

/*
 * Runtime copy of the constants the reference hard-codes at the top of main()
 * (periodicFFT/pf3d.cpp:35-73, cosFFT/mesabi/cosNoAdvMorph.cpp:74-112).
 * dx = L/N = 2 pi / (q0 Nw) in the reference.
 */
typedef struct sh_params {
  int n;             /* grid points per side: 16, 32, 64, 128, 256 or 512   */
  int batch;         /* independent replicas integrated together (>= 1)     */
  int boundary;      /* SH_PERIODIC / SH_NEUMANN                             */
  int advection;     /* 1: Stokes advection (periodic: pf3d.cpp:399-465; Neumann:
                        the sine-transform velocity of cosFFT/comet/morphSurfK.cpp) */
  int nonlinearity;  /* SH_QUINTIC / SH_QUAD_CUBIC                           */
  int scheme;        /* SH_CNAB2 / SH_IMEX_EULER                             */
  int precision;     /* SH_FP64 / SH_FP32                                    */
  int l1_interval;   /* steps between L1 evaluations (pf3d.cpp:489: 100); 0 = off */
  int energy_trace;  /* 1: record the energy of every new state              */
  int variant;       /* plane-pass cluster size (0 = default; built: 1, 2 at 64^3;
                        1, 2, 4 at 128^3; 4, 8, 16 at 256^3; 16 at 512^3)     */
  double dx, dt, eps, beta, gamma, alpha, q0, eta, rho;
  double w_mid;      /* pinning penalty weight (periodicFFT/pf3dMorph.cpp:102) */
  double sub_sigma;  /* substrate penalty sigma (cosFFT/comet/cosNoAdvMorph.cpp:67-74) */
  double sub_z0;
  const double* eps_per_replica; /* NULL, or `batch` values of epsilon       */
  int curvature;     /* Neumann curvature pass: SH_CURV_DIFFERENCE / SH_CURV_SPECTRAL */
  int replica_block; /* batched plain steps: replicas advanced together, 16 steps at a
                        time, while their state stays in L2 (0 = all replicas each step) */
  int pencil_tile;   /* lines per CTA of the pencil (x) pass: 0 = the default (16 FP32,
                        8 FP64); 8, 16 and 32 are built at 64^3 and at 128^3 with
                        variant 0 or 1 */
} sh_params;

typedef struct sh_handle sh_handle;

/* Fill `p` with the plain periodic 128^3 case (eps=-0.75, beta=2, gamma=1,
 * alpha=q0=1, dx=2 pi/8, dt=0.05, FP64, CNAB2, quintic). */
int sh_default_params(sh_params* p);

/* Allocate a solver.  Replaces the set-up part of main(): wavenumbers
 * (periodicFFT/pf3d.cpp:162-190), operator tables (:195-222, recomputed from
 * indices on the device) and the FFTW plans (:226-291). */
int sh_create(const sh_params* p, sh_handle** out);
int sh_destroy(sh_handle* h);

/* Load psi^0 for all replicas (batch * N^3 values, replica-major) and compute
 * the first N-hat (Euler start, periodicFFT/pf3d.cpp:363-374). */
int sh_set_psi(sh_handle* h, const double* host_psi, int layout);
/* Same, from a device buffer of batch*N^3 doubles (dense layout). */
int sh_set_psi_device(sh_handle* h, const double* dev_psi);
/* Copy the current psi out (gathered psi, periodicFFT/pf3d.cpp:554-568). */
int sh_get_psi(sh_handle* h, double* host_psi, int layout);
int sh_get_psi_device(sh_handle* h, double* dev_psi);

/* Advance every replica by `nsteps` time steps (the body of the while loop,
 * periodicFFT/pf3d.cpp:390-550; cosFFT/mesabi/cosNoAdvMorph.cpp:483-620).
 * Returns after the steps completed; SH_ENONFINITE if psi became NaN/Inf. */
int sh_step(sh_handle* h, int nsteps);
/* Enqueue `nsteps` steps on the handle's stream and return immediately. */
int sh_step_async(sh_handle* h, int nsteps);

/* Build ahead of time what sh_step_async replays for runs of 16 steps or
 * more without an energy trace (energy_trace = 0): a CUDA graph of 16 steps,
 * instantiated once per handle; with the L1 monitor on it replays the chunks
 * between the monitored steps (replica blocks: only with l1_interval = 0).  Runs nothing and
 * changes no state; without this call the first such sh_step builds it.  No
 * counterpart in the reference, whose loop has no set-up beyond its FFTW plans. */
int sh_prepare(sh_handle* h);

/* One drop-in time loop with host buffers: psi0 in, nsteps steps, psi out. */
int sh_run(sh_handle* h, const double* host_psi0, int nsteps, double* host_psi_out, int layout);

/* Lyapunov energy of the current state, one value per replica
 * (energyPsi.m:225-234 with the exact spectral Laplacian, FP64 sums). */
int sh_energy(sh_handle* h, double* out);
/* Dominant layer wavenumber of the current state, one value per replica: |q|
 * of the |k| shell (width 2 pi/L periodic, pi/L Neumann; shell index = the
 * rounded length of the mode's index vector) that holds the most spectral
 * power, the k = 0 shell excluded; the lowest shell wins a tie.  The power of
 * each mode is |psihat|^2 of the R2C spectrum (each kz in (0, N/2) counted
 * twice for its conjugate) or of the REDFT10 spectrum (halved on each zero
 * index), summed per shell in FP64.  The quantity pf3dVal's sweep probes
 * (periodicFFT/pf3dVal.cpp:214-325) for long runs. */
int sh_dominant_wavenumber(sh_handle* h, double* out);
/* Stokes velocity of the current state of an advected handle (advection = 1),
 * batch*N^3 doubles per component, dense (i, j, k) order.  Periodic: the
 * Fourier solve of periodicFFT/pf3d.cpp:399-451.  Neumann: the sine-transform
 * solve of cosFFT/comet/morphSurfK.cpp:686-882 (S = (L psi) grad psi with
 * difference gradients one-sided at the walls, RODFT10, the projector with the
 * sine wavenumbers pi (m+1)/L, RODFT01), which morphSurfK computes but does
 * not use or write. */
int sh_velocity(sh_handle* h, double* ux, double* uy, double* uz);
/* Energies recorded by energy_trace: out[s*batch + r] for the first
 * min(max_steps, steps taken) steps; *count receives the number of steps. */
int sh_energy_trace(sh_handle* h, double* out, int max_steps, int* count);
/* Latest L1 monitor values (periodicFFT/pf3d.cpp:489-509), one per replica,
 * and how many evaluations happened so far. */
int sh_l1(sh_handle* h, double* out, int* count);

/* Surface pass, one step.  Writes N*N values per replica in (i, j) order:
 * z index (or -1), v_n, H, K (NaN where no crossing).
 * Periodic, advected handles: surfTrack (periodicFFT/surfTrack.cpp:602-626,
 *   767-806): takes one step and scans every column of the new psi (+z, first
 *   psi < 0 after psi > 0.1).
 * Neumann handles: the curvature pass of cosFFT/comet/cosNoAdvMorphCurv.cpp:
 *   742-965 at the current state (spectral psi_xx, psi_yy, psi_zz and d_t psi,
 *   difference gradients, -z scan for the first psi < 0 after psi > 0.7,
 *   Megrabov's H and K), then takes one step. */
int sh_surface_step(sh_handle* h, int* z, double* vn, double* hmean, double* kgauss);

/* Local-amplitude map of the current psi (cosFFT/comet/morphSurfAmp.cpp:
 * 1005-1125): psiAvg = trapezoid integral of psi^2 over the box of +-Nw/2
 * cells around each point (clipped at the grid edge), divided by the same
 * integral over the box [Nw/2, 3 Nw/2]^3 times the box volume / (2 pi/q0)^3.
 * Writes N^3 doubles per replica, dense (i, j, k) order.  Needs
 * 3 (Nw/2) <= N - 1. */
int sh_local_amplitude(sh_handle* h, int nw, double* out);

/* Discrete adjoint of the CNAB2 loop (plain periodic step, SH_CNAB2, no
 * advection or penalty).  Integrates `nsteps` steps from psi0, then runs the
 * reverse sweep for a loss L whose gradient with respect to psi^T is
 * dl_dpsi_t (e.g. psi^T - target for 1/2 ||psi^T - target||^2), recomputing
 * the forward states from checkpoints taken every `ckpt_every` steps.
 * Outputs per replica: dL/d eps, dL/d q0 (FP64 accumulation) and dL/d psi0
 * (batch*N^3).  No counterpart in the reference (a differentiation
 * addition); the forward pass is the reference loop (periodicFFT/pf3dVal.cpp:270-301). */
int sh_adjoint(sh_handle* h, const double* psi0, int nsteps, const double* dl_dpsi_t, int ckpt_every,
               double* g_eps, double* g_q0, double* g_psi0);

/* The two halves of sh_adjoint, for callers that want psi^T before they know
 * the loss (an autograd forward, then its backward).  sh_adjoint_forward sets
 * psi0, takes nsteps steps keeping a checkpoint every ckpt_every steps, and
 * leaves the handle at psi^T (read it with sh_get_psi).  sh_adjoint_backward
 * runs the recompute and reverse sweep from those checkpoints for the loss
 * gradient dl_dpsi_t at psi^T; the handle must still hold the state the
 * forward sweep ended in (any step, sh_set_psi or sh_checkpoint_load in
 * between returns SH_ESTATE), and is left in it, so several losses can be
 * differentiated after one forward sweep. */
int sh_adjoint_forward(sh_handle* h, const double* psi0, int nsteps, int ckpt_every);
int sh_adjoint_backward(sh_handle* h, const double* dl_dpsi_t, double* g_eps, double* g_q0, double* g_psi0);

/* Binary checkpoint of the full state (including the AB2 history, which the
 * reference's text files drop): query size with buf == NULL. */
int sh_checkpoint_save(sh_handle* h, void* buf, size_t* bytes);
int sh_checkpoint_load(sh_handle* h, const void* buf, size_t bytes);

/*
 * L1 monitor of two device psi fields that allocates no device memory.
 * No counterpart in the reference. It computes, per replica,
 *   L1 = sum |psi_new - psi_old| / (dt sum |psi_new|),
 * the relaxation monitor that sh_l1 reports, on buffers the caller owns. It
 * is for callers that must not let a library allocate. Examples: a host that
 * manages all device memory through its own pool, and real-time loops that
 * cannot take the implicit device synchronisation of cudaMalloc/cudaFree.
 *
 * dev_psi_new, dev_psi_old: batch*n3 doubles each on the current device.
 * dev_out: batch doubles on the current device; receives L1 per replica.
 * stream: a cudaStream_t; the call is stream-ordered and returns without
 * synchronising.
 *
 * The per-block partial sums go into one fixed device array of the library
 * (256 KiB, held by every GPU that loads the library until the process
 * exits). batch is therefore at most SH_L1_NOALLOC_MAX_BATCH; larger values
 * return SH_EINVAL. The first call on a device looks up that array's device
 * address (cudaGetSymbolAddress) with the device current and keeps it for the
 * rest of the process. Make that first call before any stream capture. A
 * cudaDeviceReset discards the array with the rest of the device state, so
 * the kept address is stale afterwards: do not call this entry point on a
 * device after resetting it. Each call overwrites every slot it reads, so no
 * state carries over between calls. Calls that overlap on the GPU (on
 * different streams, or on several host threads) share the array and race.
 * Errors: sh_last_error(NULL).
 */
#define SH_L1_NOALLOC_MAX_BATCH 128
int sh_l1_noalloc(const double* dev_psi_new, const double* dev_psi_old, long long n3, int batch, double dt,
                  double* dev_out, void* stream);

/* Pinned host memory for fast host<->device copies. */
int sh_host_alloc(size_t bytes, void** out);
int sh_host_free(void* p);

/* Run `nsteps` steps timing every kernel launch with CUDA events; returns
 * the summed device milliseconds of the pencil (x) and plane (y,z) passes. */
int sh_profile_steps(sh_handle* h, int nsteps, double* ms_pencil, double* ms_plane);

/* Residency of the two step kernels on the handle's GPU, written to out[7]:
 *   out[0] plane-pass CTAs per SM, out[1] plane clusters resident at once,
 *   out[2] plane cluster size (CTAs), out[3] plane CTAs in one pass,
 *   out[4] pencil-pass CTAs per SM, out[5] pencil CTAs in one pass,
 *   out[6] SM count.
 * A pass of G CTAs runs in G / (resident CTAs) waves; when that is not a
 * whole number the last wave leaves SMs idle.  Allocates nothing. */
int sh_residency(sh_handle* h, int* out);

int sh_synchronize(sh_handle* h);
void* sh_stream(sh_handle* h);               /* the handle's cudaStream_t (NULL handle: NULL) */
long long sh_steps_taken(sh_handle* h);      /* steps since sh_set_psi, or as restored by sh_checkpoint_load (NULL handle: -1) */
int sh_kernel_launches(sh_handle* h, long long* count);
const char* sh_last_error(sh_handle* h);     /* NULL handle: last global error */
const char* sh_version(void);

#ifdef __cplusplus
}
#endif
#endif /* SMECTIC_B200_H */
