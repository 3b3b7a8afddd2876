/*
 * lcs_b200.h -- C ABI of the B200 time-step backend for LCS.jl.
 *
 * The reference plugs a backend into `LCS.simulate` by Julia dispatch on the
 * backend type: `LCS.timestep!` (src/simulate.jl:55) and `LCS.evolve!`
 * (src/simulate.jl:56) are the two per-step calls, and below them the stage
 * functions `Flows.rhs!/update!/couple!/forcing!/timestep` and
 * `Particles.boundary!/motion!/update!/timestep`.  A Julia package `LCSB200`
 * binds the entry points below with `ccall`; everything else (config, init,
 * stats, HDF5 I/O) stays in the reference's own Julia code on the host.
 *
 * Conventions
 *  - Every call returns LCS_OK (0) or a negative LCS_E* code; the message is
 *    available from lcs_last_error(h) (or lcs_last_error(NULL) when
 *    lcs_create itself failed).  Nothing throws or aborts across the ABI.
 *  - Host arrays are caller-owned, FP64, x fastest (Julia column-major, so a
 *    Julia `Array{Float64,3}` of size (nx,ny,nz) is bit-for-bit the C array
 *    [nz][ny][nx]); they are only read or written during the call.
 *  - "interior" arrays hold the n^3 cells 1..n of each axis (`LCS.unhalo`,
 *    src/config.jl:114-118); "haloed" arrays hold (n+2h)^3 cells with logical
 *    index i in 1-h..n+h at offset i+h-1 (`@offsetviews`,
 *    lib/offsets/src/Offsets.jl:70-73).
 *  - A handle owns all device memory and one CUDA stream.  It is used by one
 *    host thread at a time; distinct handles are independent.
 *  - Stage arguments are 1 or 2 (`LCS.RKStage1/RKStage2`, src/rungekutta.jl).
 *    Stage functions take the stage time increment `dtrk` the reference passes
 *    them (`LCS.dtrk`, src/state.jl:37-38: dt/2 in stage 1, dt in stage 2).
 */
#ifndef LCS_B200_H
#define LCS_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define LCS_API __attribute__((visibility("default")))
#else
#define LCS_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define LCS_ABI_VERSION 1
#define LCS_MAX_SPECIES 16

/* ---- status codes ------------------------------------------------------ */
#define LCS_OK 0
#define LCS_EINVAL (-1)      /* bad config or argument (reference: ArgumentError) */
#define LCS_ENOMEM (-2)      /* device memory / pool budget exhausted */
#define LCS_ECUDA (-3)       /* a CUDA runtime call failed */
#define LCS_ETIMEDOUT (-4)   /* a bounded device wait gave up */
#define LCS_ENONFINITE (-5)  /* NaN/Inf residual or dt */
#define LCS_ESTATE (-6)      /* call out of order (e.g. evolve before upload) */

/* ---- config enums (PolySerde kinds of the reference) ------------------- */
enum lcs_mode { LCS_MODE_FLOW = 0, LCS_MODE_FLOW_PARTICLE = 1 };      /* src/config.jl:1-20 */
enum lcs_coloring {                                                   /* lib/parallel/src/foraxes.jl */
  LCS_COLORING_NO = 0,             /* NoColoring (:51) -- racy on a GPU, rejected */
  LCS_COLORING_RED_BLACK = 1,      /* RedBlack (:82-88) */
  LCS_COLORING_RED_BLACK_FAST = 2, /* RedBlackFast (:93-107) */
  LCS_COLORING_RED_BLACK_BLOCK = 3 /* RedBlackBlock(size) (:114-136) */
};
enum lcs_forcing {                 /* src/flows/config.jl:100-175 */
  LCS_FORCING_NO = 0,              /* "no" */
  LCS_FORCING_LINEAR_POWER = 1,    /* "linear-power" ConstantPowerLF */
  LCS_FORCING_RC_ENERGY = 2        /* "rc-energy" EnergyPreserveRCF */
};
enum lcs_drag { LCS_DRAG_LINEAR = 0, LCS_DRAG_NONLINEAR = 1 };        /* src/particles/config.jl:118-139 */
enum lcs_precision {
  LCS_PRECISION_FP64 = 0,          /* the reference's arithmetic (const FP = Float64, src/LCS.jl:20) */
  LCS_PRECISION_FP32_MIXED = 1     /* FP32 fields; FP64 residuals, energies, positions (no reference counterpart) */
};

/* Field identifiers for lcs_field_set/get (src/flows/buffer.jl:38-58). */
enum lcs_field {
  LCS_FIELD_U = 0, LCS_FIELD_V = 1, LCS_FIELD_W = 2,    /* Us   (haloed) */
  LCS_FIELD_U2 = 3, LCS_FIELD_V2 = 4, LCS_FIELD_W2 = 5, /* Us2  (haloed) */
  LCS_FIELD_P = 6,                                      /* P    (haloed) */
  LCS_FIELD_DUDT = 7, LCS_FIELD_DVDT = 8, LCS_FIELD_DWDT = 9 /* dUdts (interior only) */
};

/* Particle property identifiers (src/particles/buffer.jl:1-37). */
enum lcs_prop {
  LCS_PROP_X = 0, LCS_PROP_Y, LCS_PROP_Z,          /* xss   */
  LCS_PROP_X2, LCS_PROP_Y2, LCS_PROP_Z2,           /* xss2  */
  LCS_PROP_U, LCS_PROP_V, LCS_PROP_W,              /* uss   */
  LCS_PROP_U2, LCS_PROP_V2, LCS_PROP_W2,           /* uss2  */
  LCS_PROP_DUDT, LCS_PROP_DVDT, LCS_PROP_DWDT,     /* dudtss */
  LCS_PROP_DIAM,                                   /* diams */
  LCS_NPROP
};

/* One particle species (`ParticleConfig`, src/particles/config.jl:35-41,
 * 118-139, 11-24).  Diameters are per particle and uploaded. */
typedef struct lcs_species {
  int64_t nvalid;        /* particles of this species on the device */
  double gravity;        /* ParticleParams.gravity (acts on x, motion.jl:77) */
  double density_ratio;  /* ParticleParams.density_ratio */
  int32_t drag;          /* enum lcs_drag */
  int32_t _pad;
} lcs_species;

/* POD mirror of `LCS.Config` restricted to what the time step reads. */
typedef struct lcs_config {
  int32_t abi_version;   /* = LCS_ABI_VERSION */
  int32_t mode;          /* enum lcs_mode */
  int32_t dims[3];       /* Grid.dims (cubic, even) */
  int32_t halo_size;     /* Grid.halo_size (>= 3 for time blocking; >= 2 otherwise) */
  double cfl, dtmax;     /* TimeStep */
  double U0, L0, NU;     /* FlowParams (Re = U0*L0/NU) */
  /* HSMAC (src/flows/config.jl:88-98) */
  int32_t time_blocking, overlap, coloring, coloring_block;
  double omega, epsp;
  int32_t itrmin, itrmax;
  /* forcing */
  int32_t forcing;       /* enum lcs_forcing */
  int32_t kmin, kmax, coarse_size;   /* rc-energy */
  double power;          /* linear-power P0 */
  double energy;         /* rc-energy e10 */
  /* particles */
  int32_t n_species;
  int32_t precision;     /* enum lcs_precision */
  lcs_species species[LCS_MAX_SPECIES];
  int32_t device;        /* CUDA device ordinal */
  int32_t use_graphs;    /* 1: lcs_step runs device-resident CUDA graphs */
} lcs_config;

/* Per-couple log `(; itr, div)` (src/flows/couples/hsmac.jl:128,200). */
typedef struct lcs_couple_log { int32_t itr; int32_t sweeps; double div; } lcs_couple_log;

/* The log NamedTuple of one `evolve!` (src/evolve.jl:124-145). */
typedef struct lcs_log {
  lcs_couple_log couple1, couple2;
  double forcing_p;      /* (; p) of the forcing, NaN for "no" */
  double forcing_e10;    /* (; e10) of rc-energy, NaN otherwise */
  double dt;             /* dt used by this step */
  double t;              /* time after the step */
  int64_t step;          /* step after the step */
} lcs_log;

typedef struct lcs_handle lcs_handle;

/* ---- lifetime ---------------------------------------------------------- */
/* Replaces `LCS.Buffer(config, topo)` + `LCS.State` (src/buffer.jl:27-34, src/state.jl:27-35). */
LCS_API int lcs_create(const lcs_config* cfg, lcs_handle** out);
LCS_API void lcs_destroy(lcs_handle* h);
LCS_API const char* lcs_last_error(const lcs_handle* h);
/* The configuration the handle was created with. */
LCS_API int lcs_get_config(const lcs_handle* h, lcs_config* out);
/* Bytes of device memory the handle holds (the serving admission uses it). */
LCS_API int lcs_footprint(const lcs_config* cfg, int64_t* bytes);
/* The device's FP64 FMA throughput in TFLOP/s, measured with a kernel of
 * independent fused multiply-add chains (the denominator of the FP64
 * roofline of compute-heavy kernels such as rhs!). */
LCS_API int lcs_measure_fp64_peak(int32_t device, double* tflops);

/* ---- state transfer (host FP64 in every precision form) ---------------- */
/* Interior U,V,W,P in, halos left for the next synchalo (src/flows/inits/init.jl). */
LCS_API int lcs_upload_flow(lcs_handle* h, const double* U, const double* V, const double* W, const double* P);
LCS_API int lcs_download_flow(lcs_handle* h, double* U, double* V, double* W, double* P);
/* The `upsample` init (src/LCSIO/upsample.jl:1-91, flows/config.jl:58-64):
 * coarse interiors of (nx/2, ny/2, nz/2) cells, as read from a coarse restart,
 * periodically extended by one cell and trilinearly upsampled 2x into the
 * interior of U, V, W and P (trilinear_upsample2x!, upsample.jl:47-91).  Dims
 * must be even; halos are left for the next synchalo. */
LCS_API int lcs_upload_flow_coarse(lcs_handle* h, const double* U, const double* V, const double* W, const double* P);
/* Whole field, interior (haloed=0) or haloed (haloed=1) layout. */
LCS_API int lcs_field_set(lcs_handle* h, int32_t field, const double* data, int32_t haloed);
LCS_API int lcs_field_get(lcs_handle* h, int32_t field, double* data, int32_t haloed);
/* All valid particles of one species (src/particles/init.jl). ids may be NULL. */
LCS_API int lcs_upload_particles(lcs_handle* h, int32_t species, int64_t n, const int64_t* ids, const double* diam,
                         const double* x, const double* y, const double* z,
                         const double* u, const double* v, const double* w);
LCS_API int lcs_download_particles(lcs_handle* h, int32_t species, int64_t* ids, double* diam,
                           double* x, double* y, double* z, double* u, double* v, double* w);
LCS_API int lcs_prop_set(lcs_handle* h, int32_t species, int32_t prop, const double* data);
LCS_API int lcs_prop_get(lcs_handle* h, int32_t species, int32_t prop, double* data);
/* State (step, t) as `LCS.State` holds it. */
LCS_API int lcs_set_state(lcs_handle* h, int64_t step, double t);
LCS_API int lcs_get_state(lcs_handle* h, int64_t* step, double* t);

/* ---- the per-step calls ------------------------------------------------ */
/* `LCS.timestep` (src/timestep.jl:14-27): min(Flows.timestep, Particles.timestep). */
LCS_API int lcs_timestep(lcs_handle* h, double* dt);
/* `LCS.evolve!` (src/evolve.jl:15-146) with state.dt = dt; fills *log if non-NULL. */
LCS_API int lcs_evolve(lcs_handle* h, double dt, lcs_log* log);
/* nsteps x (timestep! + evolve!) with no host round trip in between;
 * logs[nsteps] may be NULL. */
LCS_API int lcs_step(lcs_handle* h, int32_t nsteps, lcs_log* logs);
/* lcs_step, with the device time of the nsteps measured by CUDA events
 * recorded on the handle's stream before the first and after the last step. */
LCS_API int lcs_step_timed(lcs_handle* h, int32_t nsteps, lcs_log* logs, double* device_ms);

/* ---- stage functions (one reference function each) -------------------- */
/* `Topologies.synchalo!(FullHalo(r) | FaceHalo(r), fields)` single process
 * (lib/topologies/src/halo.jl:138-159).  fields is a bitmask of 1<<lcs_field. */
LCS_API int lcs_synchalo(lcs_handle* h, int32_t field_mask, int32_t r, int32_t full);
/* `Flows.rhs!` (src/flows/rhs.jl:20-42) on Us_rhs(stage) -> dUdts. */
LCS_API int lcs_flow_rhs(lcs_handle* h, int32_t stage);
/* `Flows.update!` (src/flows/update.jl:23-54): Us_update(stage) = Us0 + dUdts*dtrk. */
LCS_API int lcs_flow_update(lcs_handle* h, int32_t stage, double dtrk);
/* rhs! then update! fused in one pass (dUdts is not written). */
LCS_API int lcs_flow_rhs_update(lcs_handle* h, int32_t stage, double dtrk);
/* `Flows.couple!(::HSMAC)` (src/flows/couples/hsmac.jl:52-75) on Us_couple(stage). */
LCS_API int lcs_flow_couple(lcs_handle* h, int32_t stage, double dtrk, lcs_couple_log* log);
/* `Flows.forcing!` stage 2 (src/flows/forcings/{lf,rcf}.jl) on Us; p and e10 out. */
LCS_API int lcs_flow_forcing(lcs_handle* h, double dtrk, double* p, double* e10);
/* `Flows.timestep` (src/flows/timestep.jl:18-65), including its FaceHalo sync. */
LCS_API int lcs_flow_timestep(lcs_handle* h, double* dt);
/* `Particles.timestep` (src/particles/timestep.jl:6-25) over all species. */
LCS_API int lcs_particles_timestep(lcs_handle* h, double* dt);
/* `Particles.boundary!` periodic part (src/particles/boundary.jl:33-120). */
LCS_API int lcs_particles_boundary(lcs_handle* h, int32_t species, int32_t stage);
/* `Particles.motion!` (src/particles/motion.jl:10-84). */
LCS_API int lcs_particles_motion(lcs_handle* h, int32_t species, int32_t stage);
/* `Particles.update!` (src/particles/update.jl:19-65). */
LCS_API int lcs_particles_update(lcs_handle* h, int32_t species, int32_t stage, double dtrk);
/* New init kind (no reference counterpart): particle velocity = the trilinear
 * interpolation (src/particles/interp.jl:62-126) of the current Us at xss. */
LCS_API int lcs_init_particle_velocity(lcs_handle* h, int32_t species);

/* ---- profiling (`LCS_LOG_LEVEL=PROFILE`, src/log.jl:6-20) --------------- */
/* When enabled, every kernel launch is bracketed by CUDA events on the
 * handle's stream; totals are per kernel label. */
LCS_API int lcs_profile_enable(lcs_handle* h, int32_t on);
LCS_API int lcs_profile_reset(lcs_handle* h);
LCS_API int lcs_profile_count(lcs_handle* h, int32_t* n);
LCS_API int lcs_profile_entry(lcs_handle* h, int32_t i, char* name, int32_t name_cap, double* total_ms, int64_t* launches);
/* Number of this library's kernel launches since creation (or the last reset). */
LCS_API int lcs_launch_count(lcs_handle* h, int64_t* launches);
/* Bytes this handle copied host->device and device->host since creation. */
LCS_API int lcs_transfer_stats(lcs_handle* h, int64_t* h2d_bytes, int64_t* d2h_bytes);
LCS_API int lcs_synchronize(lcs_handle* h);

/* ---- statistics ----------------------------------------------------------
 * `Flows.stat` (src/flows/stat.jl:66-153) on the device, on Us: the Summary
 * (mean, max, min) of U, V, W, and k, epsilon, tau_eta, lambda (l_mu), l_eta,
 * Re_lambda, u' (urms), k_eta, skewness and flatness of du/dx.  Reductions in
 * FP64 in both precision forms; the halo is read through periodic wrapping, so
 * the call changes no state.  The integral length L and C_epsilon are 0, as in
 * the reference without an integral-length buffer (stat.jl:155). */
typedef struct lcs_flow_stats {
  double u_mean, u_max, u_min, v_mean, v_max, v_min, w_mean, w_max, w_min;
  double k, epsilon, tau_eta, l_mu, l_eta, Re_lambda, urms, k_eta, skewness, flatness, L, C_epsilon;
} lcs_flow_stats;
LCS_API int lcs_flow_stat(lcs_handle* h, lcs_flow_stats* out);
/* Divergence of the current velocity over the n^3 interior cells, in the
 * HSMAC form (hsmac.jl: dxi (U[i]-U[i-1]) + dyi (V[j]-V[j-1]) + dzi
 * (W[k]-W[k-1]), periodic): its RMS and its max |div| (a diagnostic beside the
 * couple log's residual, which the reference takes over 1:n+1). */
LCS_API int lcs_flow_divergence(lcs_handle* h, double* rms, double* maxabs);
/* Test hook for the bounded device waits (no reference counterpart; the
 * reference has no device-side waits).  kind 1 makes the grid barriers of the
 * cooperative face-phase kernel of overlap sweeps wait for one arrival more
 * than there are blocks; kind 2 makes the row-warp sweep's TMA plane barriers
 * expect 16 bytes more than its copies deliver.  The next launch that waits
 * then runs its wait out at the bound (about 0.1 s for a grid barrier, 2^22
 * polls for a plane barrier; the sweep still waits, bounded, for the copies
 * it issued before it returns), sets the handle's sticky wait error and stops
 * the couple: the call returns LCS_ETIMEDOUT and so does every later step of
 * the handle.  kind 0 (the default) restores normal waits; the handle stays
 * failed and is destroyed.  No trap, no hang: the context stays usable for
 * other handles. */
LCS_API int lcs_debug_unreachable_waits(lcs_handle* h, int32_t kind);

/* `Particles.makeindex!` (src/particles/makeindex.jl:29-67) on species s with
 * the positions of stage (1: xss, 2: xss2): cell index ci = floor(x / dxc) + 1
 * per axis (dxc = (2pi/n) * grid_ratio, particles/config.jl:60), hash = the
 * 1-based column-major index of ci over the cell axes 0:nc+1 (nc = n /
 * grid_ratio), a stable sort of the species' particles by hash that permutes
 * every property (the device order of the species changes; ids follow), and
 * starts/stops of every hash 1..(nc+2)^3 (src/utils/fast.jl:8-40). */
LCS_API int lcs_particles_makeindex(lcs_handle* h, int32_t species, int32_t stage, int32_t grid_ratio);
/* Keep the particles in cell order (no reference counterpart): after every
 * step of lcs_step or lcs_step_begin that brings the step counter to a
 * multiple of `interval`, makeindex! (as lcs_particles_makeindex, stage 1,
 * this grid_ratio) runs on every species.  The fluid gathers of motion! then
 * read neighbouring cells together.  Each particle's arithmetic does not depend
 * on its place in the arrays, so a particle's values (matched by id) are those
 * of the unsorted run, bit for bit; only the order changes.  interval = 0
 * turns it off (the default).  lcs_evolve does not sort: a caller stepping
 * with lcs_timestep/lcs_evolve calls lcs_particles_makeindex itself.  Steps of
 * a batch group (lcs_group_step_begin) sort each member that has a sort, on
 * the group's stream between the group's step graphs. */
LCS_API int lcs_set_particle_sort(lcs_handle* h, int32_t interval, int32_t grid_ratio);
/* The last cell index of species s: hashes[nvalid], starts[(nc+2)^3],
 * stops[(nc+2)^3] (Int64, as LCS.IP); NULL pointers are skipped. */
LCS_API int lcs_particles_cellindex(lcs_handle* h, int32_t species, int64_t* hashes, int64_t* starts, int64_t* stops);

/* `Particles.stat` (src/particles/stat.jl:113-151) of species s: Summary
 * (mean, max, min; src/stat.jl:20-22) of xss, uss and diams, taup of the mean
 * diameter (config.jl:41), St = taup / tau_eta (tau_eta of the flow's stat,
 * lcs_flow_stat), then makeindex! on xss (the species is reordered, as in the
 * reference), the radial distribution function of rdf_assume_ci
 * (src/particles/rdf.jl:1-103) and the number-density spectrum
 * (src/particles/spectrum.jl:11-78).  The configuration mirrors Cell, RDF and
 * Spectrum (src/particles/config.jl:51-94). */
#define LCS_RDF_MAX_BINS 1024
#define LCS_SPECTRUM_MAX_SHELLS 19 /* the WAVENUMBERS table, spectrum.jl:1 */
#define LCS_SPECTRUM_MAX_SAMPLES 1024
typedef struct lcs_particle_stat_config {
  int32_t grid_ratio;        /* Cell.grid_ratio */
  int32_t bin_size;          /* RDF.bin_size: number of bins, 1..LCS_RDF_MAX_BINS */
  int32_t search_cell_size;  /* RDF.search_cell_size */
  int32_t max_wavenumber;    /* Spectrum.max_wavenumber */
  int32_t nsamples;          /* Spectrum.nsamples: directions, 2..LCS_SPECTRUM_MAX_SAMPLES */
  int32_t pad_;
  double contact_tolerance;  /* RDF.contact_tolerance */
  double min_radius;         /* RDF.min_radius */
} lcs_particle_stat_config;
typedef struct lcs_summary {
  double mean, max, min;
} lcs_summary;
typedef struct lcs_particle_stats {
  lcs_summary x, y, z, u, v, w, diam;
  double taup, St;
  /* RDFStat (stat.jl:30-38): edges[nbins+1] are logrange(min_radius,
   * search_cell_size * min spacing, nbins + 1) */
  double gr_contact;
  int64_t npairs_contact;
  int32_t nbins, nshells;
  double edges[LCS_RDF_MAX_BINS + 1];
  double gr[LCS_RDF_MAX_BINS];
  int64_t npairs[LCS_RDF_MAX_BINS];
  /* SpectrumStat (stat.jl:10-15) */
  double wavenumbers[LCS_SPECTRUM_MAX_SHELLS];
  double Enp[LCS_SPECTRUM_MAX_SHELLS];
} lcs_particle_stats;
LCS_API int lcs_particles_stat(lcs_handle* h, int32_t species, const lcs_particle_stat_config* cfg, double tau_eta,
                               lcs_particle_stats* out);
/* `Particles.density` (src/particles/stat.jl:176-215): makeindex! on xss
 * (reorders the species), then per particle the cubic-spline SPH sum over the
 * 27 neighbouring cells with h = min spacing; densities[nvalid] in the new
 * device order (0 for a particle outside the cell domain). */
LCS_API int lcs_particles_density(lcs_handle* h, int32_t species, int32_t grid_ratio, double* densities);

/* ---- restart files (src/LCSIO/save.jl:40-167, load.jl:23-118) ------------
 * The reference's restart layout in HDF5 (written and read without an HDF5
 * library, for the subset these files use: version 0 superblock, symbol-table
 * groups, contiguous little-endian F64/I64 datasets):
 *   /flow/{U,V,W,P}                        Float64 (nz, ny, nx), the interiors
 *   /particles/<s+1>/counts                Int64 (1,) = nvalid
 *   /particles/<s+1>/{id,x,y,z,u,v,w,diam} Int64 / Float64 (nvalid,)
 * lcs_restart_load reads such a file into the handle (its dims and particle
 * counts must match, as load.jl checks); lcs_restart_load_coarse reads the
 * flow of a restart with half the dims and upsamples it (the `upsample` init,
 * src/LCSIO/upsample.jl:1-45).  lcs_stat_state_save/load write and read the
 * `<step>/state/{step,t,dt}` entries of a stat file (save.jl:17-31, the resume
 * of load.jl:1-21).  lcs_h5_dataset / lcs_h5_list inspect any file of the
 * subset.  Errors: LCS_EINVAL with lcs_io_last_error(). */
LCS_API int lcs_restart_save(lcs_handle* h, const char* path);
LCS_API int lcs_restart_load(lcs_handle* h, const char* path);
LCS_API int lcs_restart_load_coarse(lcs_handle* h, const char* path);
LCS_API int lcs_stat_state_save(const char* path, int64_t step, double t, double dt);
/* One `<step>` entry of the stat file as `LCSIO.savestat` (save.jl:1-33)
 * writes it with Utils.deepwrite (src/utils/hdf5.jl:5-19), the Julia field
 * names as dataset names (UTF-8), scalars as rank-0 datasets:
 *   <step>/state/{step,t,dt}, <step>/state/particles/<s+1>/nvalid
 *   <step>/stat/state/{step,t,dt}
 *   <step>/stat/flow/{u,v,w}/{mean,max,min}, k, ϵ, τη, lμ, lη, Reλ, urms, kη,
 *        skew, flat, L, Cϵ                        (FlowStat, flows/stat.jl:22-39)
 *   <step>/stat/particles/<s+1>/{x,y,z,u,v,w,diam}/{mean,max,min}, τp, St,
 *        rdf/{gr_contact,npairs_contact,edges,gr,npairs},
 *        spectrum/{wavenumbers,Enp}               (particles/stat.jl:10-77)
 *   <step>/log/flow/couple{1,2}/{itr,div}, <step>/log/flow/forcing/{p,e10}
 * flow, nvalid, particles (n_species entries) and log may be NULL: their
 * subtrees are left out, as deepwrite writes nothing for `nothing`; empty
 * arrays and NaN forcing values are left out too.  Like the reference's "cw"
 * open, the other steps of an existing file are kept and an existing <step>
 * is replaced (lcs_stat_state_save does the same); the file is rewritten
 * through a temporary file.  A group holds at most 8192 entries. */
LCS_API int lcs_stat_save(const char* path, int64_t step, double t, double dt, const lcs_flow_stats* flow,
                          int32_t n_species, const int64_t* nvalid, const lcs_particle_stats* particles,
                          const lcs_log* log);
LCS_API int lcs_stat_state_load(const char* path, int64_t step, double* t, double* dt);
LCS_API int lcs_h5_dataset(const char* path, const char* name, int32_t* rank, int64_t* dims, char* kind, void* buf,
                           int64_t bytes);
LCS_API int lcs_h5_list(const char* path, const char* group, char* buf, int64_t cap);
LCS_API const char* lcs_io_last_error(void);

/* ---- asynchronous steps (no reference counterpart) ----------------------
 * For hosts that drive many handles at once (the batching and serving forms
 * below, or a Julia task per handle).  lcs_step_begin enqueues nsteps
 * (1..LCS_MAX_ASYNC_STEPS) device-resident steps, as lcs_step runs them, on
 * the handle's stream and returns at once; lcs_step_poll reports whether they
 * have finished without blocking; lcs_step_finish waits for them and fills
 * logs[nsteps] (may be NULL).  Between begin and finish the handle accepts no
 * other call but poll (ESTATE). */
#define LCS_MAX_ASYNC_STEPS 4096
LCS_API int lcs_step_begin(lcs_handle* h, int32_t nsteps);
LCS_API int lcs_step_poll(lcs_handle* h, int32_t* done);
LCS_API int lcs_step_finish(lcs_handle* h, lcs_log* logs);
/* Device bytes the handle holds (its pool), as lcs_footprint predicts. */
LCS_API int lcs_device_bytes(lcs_handle* h, int64_t* bytes);
/* Launch shapes of a handle, set from outside (no reference counterpart; the
 * batch's autotuner and the server use it): rw_rows = tile rows of the
 * HSMAC sweep (13, 8 or 5, or 29 in FP32: two rows a warp; 0 keeps the
 * current), zchunk = planes per z chunk
 * of a sweep (0: the built-in cost model), share = the part of the GPU the
 * handle's launches are sized for when several handles run at once (0, 1].
 * FP64 fields do not depend on these (the residual's partial sums are grouped
 * differently); the step graphs are captured again. */
LCS_API int lcs_set_tuning(lcs_handle* h, int32_t rw_rows, int32_t zchunk, double share);

/* ---- batching form (no reference counterpart) ---------------------------
 * An ensemble of independent runs with uneven grid sizes, particle counts and
 * parameters, advanced together: lcs_batch_step enqueues every member's steps
 * (each a CUDA-graph replay on the member's own stream) before waiting for any,
 * so the members' kernels overlap on the GPU.  Each member computes exactly
 * what it computes alone.  Members are ordinary handles (lcs_batch_member) for
 * uploads, downloads and single-member calls between batch steps; the batch
 * owns and destroys them.  logs is member-major: logs[i * nsteps + q].
 * lcs_batch_create and lcs_server_create set CUDA_DEVICE_MAX_CONNECTIONS=32
 * (unless already set) so that up to 32 member streams get their own hardware
 * work queue; it takes effect only if the process has no CUDA context yet. */
typedef struct lcs_batch lcs_batch;
LCS_API int lcs_batch_create(const lcs_config* members, int32_t m, lcs_batch** out);
/* A group: 2..64 handles of one shape (dims, halo, HSMAC settings, precision)
 * and one set of launch shapes (lcs_set_tuning) whose steps run as one CUDA
 * graph.  Each member's own kernels run member after member; each couple's
 * HSMAC loop is one device-side loop for the whole group whose sweep, halo and
 * face kernels are launched once for all members (a member computes exactly
 * what it computes alone with the same launch shapes).  lcs_group_step_begin
 * enqueues nsteps steps of every member; lcs_step_poll / lcs_step_finish on
 * each member then complete them as for lcs_step_begin.  The group does not
 * own its members; destroy it before them.  lcs_batch_create groups members
 * this way by itself. */
typedef struct lcs_group lcs_group;
LCS_API int lcs_group_create(lcs_handle* const* members, int32_t m, lcs_group** out);
LCS_API int lcs_group_step_begin(lcs_group* group, int32_t nsteps);
LCS_API void lcs_group_destroy(lcs_group* group);
LCS_API int lcs_batch_size(const lcs_batch* b, int32_t* m);
LCS_API int lcs_batch_member(lcs_batch* b, int32_t i, lcs_handle** h);
LCS_API int lcs_batch_step(lcs_batch* b, int32_t nsteps, lcs_log* logs);
/* The launch shapes lcs_batch_create chose for member i (see lcs_set_tuning):
 * its autotuner steps probe handles of each member shape together for every
 * candidate tile height and z chunk and keeps the fastest (probe_ms, one
 * probe step); LCS_BATCH_TUNE=0 in the environment skips the probing. */
LCS_API int lcs_batch_tuning(const lcs_batch* b, int32_t i, int32_t* rw_rows, int32_t* zchunk, double* share,
                             double* probe_ms);
LCS_API void lcs_batch_destroy(lcs_batch* b);

/* ---- serving form (no reference counterpart) ----------------------------
 * A request loop with continuous batching.  Requests (a config, its initial
 * state and a step count) are queued by lcs_server_submit.  The server's
 * scheduler thread admits queued requests, oldest first, whenever a slot is
 * free and the predicted device bytes of the admitted runs (lcs_footprint)
 * stay within hbm_budget_bytes; it keeps each admitted run's state on the
 * device, advances every admitted run by up to steps_per_slice steps at a
 * time with the asynchronous steps above (their work overlaps on the GPU),
 * and retires finished runs, whose final state it downloads, freeing their
 * memory for the next admissions.  A run gives the same result alone and in
 * the mix.  The submit copies the inputs: the caller's arrays may be freed on
 * return. */
typedef struct lcs_server lcs_server;
typedef struct lcs_server_config {
  int32_t device;
  int32_t max_active;        /* admitted runs at most (slots) */
  int32_t steps_per_slice;   /* steps enqueued per run per scheduling round (1..LCS_MAX_ASYNC_STEPS) */
  int32_t _pad;
  int64_t hbm_budget_bytes;  /* admitted runs' lcs_footprint sum at most */
} lcs_server_config;
typedef struct lcs_species_state {  /* one species' particles, n = config.species[s].nvalid */
  const int64_t* ids;              /* may be NULL: ids 1..n */
  const double *diam, *x, *y, *z, *u, *v, *w;
} lcs_species_state;
typedef struct lcs_request {
  lcs_config config;               /* use_graphs is forced on; device is the server's */
  const double *U, *V, *W, *P;     /* interior n^3 each, x fastest */
  lcs_species_state species[LCS_MAX_SPECIES];
  int32_t interp_velocity;         /* 1: particle velocity := fluid velocity at the particle */
  int32_t _pad;
  int64_t nsteps;                  /* timestep! + evolve! repetitions */
} lcs_request;
typedef struct lcs_species_out { double *x, *y, *z, *u, *v, *w; } lcs_species_out;  /* NULL: skipped */
enum lcs_request_state { LCS_REQ_QUEUED = 0, LCS_REQ_RUNNING = 1, LCS_REQ_DONE = 2, LCS_REQ_FAILED = 3 };
typedef struct lcs_server_stats {
  int64_t submitted, completed, failed, queued, active;
  int64_t bytes_in_use, peak_bytes_in_use;
  double p50_latency_s, p99_latency_s;   /* submit -> result ready, over completed requests */
  double mean_latency_s, busy_s;         /* busy_s: seconds with at least one admitted run */
} lcs_server_stats;
LCS_API int lcs_server_create(const lcs_server_config* c, lcs_server** out);
LCS_API int lcs_server_submit(lcs_server* s, const lcs_request* r, int64_t* ticket);
/* state: enum lcs_request_state; steps_done may be NULL. */
LCS_API int lcs_server_poll(lcs_server* s, int64_t ticket, int32_t* state, int64_t* steps_done);
/* Copies a finished request's final state (any pointer may be NULL; species
 * out[config.n_species]), its last step log and its latency (seconds from
 * submit to completion).  FAILED requests return their error code. */
LCS_API int lcs_server_result(lcs_server* s, int64_t ticket, double* U, double* V, double* W, double* P,
                              lcs_species_out* species, lcs_log* last_log, double* latency_s);
/* Forgets a finished request (its stored result). */
LCS_API int lcs_server_release(lcs_server* s, int64_t ticket);
LCS_API int lcs_server_stats_get(lcs_server* s, lcs_server_stats* out);
/* Blocks until every submitted request is DONE or FAILED, or timeout_s passes (ETIMEDOUT). */
LCS_API int lcs_server_drain(lcs_server* s, double timeout_s);
/* Stops the scheduler, finishing nothing further, and frees everything. */
LCS_API void lcs_server_destroy(lcs_server* s);
/* Message of the last failing server or batch call (thread-local). */
LCS_API const char* lcs_serve_last_error(void);

/* ---- allocation-free variant --------------------------------------------
 * No counterpart in the reference.  For callers that cannot let a library
 * call cudaMalloc: code recording a CUDA stream capture, or a process whose
 * device memory belongs to another allocator (a Julia CUDA.jl pool, a server
 * with a fixed per-request budget).  Computes `Flows.timestep`'s dt from U, V,
 * W device arrays the caller owns, laid out as the reference's haloed fields
 * ((n+2h)^3 FP64, x fastest; only the interior is read) and writes it to the
 * caller's device double *dt_out, on `stream` (a cudaStream_t, NULL for the
 * default stream).  It allocates nothing: its scratch is a static device array
 * of 3 * LCS_NOALLOC_MAX_PLANES doubles per GPU, held until the process exits,
 * so dims[2] may be at most LCS_NOALLOC_MAX_PLANES (larger grids get EINVAL).
 * Every call looks the array's device address up in the current context (a
 * reset context gets a new one); the first call on a device loads the module
 * and should come before any stream capture.  Every call shares the array:
 * calls that overlap on the GPU race, so serialise them on one stream.  A NaN
 * in U, V or W gives a NaN dt (Julia's maximum and min propagate NaN), which
 * the caller reads with the result; the call itself returns LCS_OK.  Errors
 * are reported through lcs_last_error(NULL). */
#define LCS_NOALLOC_MAX_PLANES 4096
LCS_API int lcs_flow_timestep_noalloc(const double* U, const double* V, const double* W, const int32_t dims[3],
                                      int32_t halo_size, double cfl, double dtmax, double Re, double* dt_out,
                                      void* stream);

#ifdef __cplusplus
}
#endif
#endif /* LCS_B200_H */
