/*
 * mpx.h -- C ABI of the B200 effective-field + Runge-Kutta engine (libmpx.so).
 *
 * The engine holds ferromagnets on one GPU and evaluates their effective field
 * (exchange, interfacial/general DMI, uniaxial anisotropy, Zeeman, FFT demag),
 * the LLG torque, and advances them with the explicit adaptive Runge-Kutta
 * methods of mumax+.  Everything crossing this boundary is plain C: integers,
 * doubles, and pointers with sizes.  No call throws or exits; every entry point
 * returns an mpx_status and mpx_last_error() gives the message of the last
 * failing call on the calling thread.
 *
 * Field arrays are structure-of-arrays float32, component-major, x fastest:
 * value(c, x, y, z) = a[c*N + x + nx*(y + ny*z)], N = nx*ny*nz.  This is the
 * layout of the reference's Field (core/field.hpp:15-130, one device array per
 * component) and of its numpy view (ncomp, nz, ny, nx) (bindings/fieldToArray.hpp:11-49).
 *
 * Reference interfaces each group of entry points replaces (paths relative to
 * the mumax-plus source tree):
 *   mpx_engine_*          World / MumaxWorld object (core/world.hpp:10-77,
 *                         physics/mumaxworld.hpp:26-202)
 *   mpx_magnet_*          MumaxWorld::addFerromagnet (physics/mumaxworld.cpp:57-80)
 *                         and the Ferromagnet parameter bag (physics/ferromagnet.hpp:26-99)
 *   mpx_eval / mpx_average / mpx_energy
 *                         FieldQuantity::eval() and average()
 *                         (core/fieldquantity.hpp:29-30, core/fieldquantity.cpp)
 *                         as wrapped by FM_FieldQuantity (physics/quantityevaluator.hpp:18-64)
 *   mpx_solver_*          TimeSolver (core/timesolver.hpp:14-89) and its Stepper::step()
 *                         (core/stepper.hpp:5-13, core/rungekutta.cpp:25-84)
 *   mpx_group_* / mpx_advance / mpx_poll
 *                         no reference counterpart: many independent solves
 *                         advanced together (batched and served forms).
 */
#ifndef MPX_H
#define MPX_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define MPX_ABI_VERSION 1

/* Status codes.  The reference raises C++ exceptions that pybind11 maps to
 * Python errors (std::invalid_argument -> ValueError, std::out_of_range ->
 * IndexError, std::runtime_error -> RuntimeError) and exits the process on CUDA
 * errors (cudautil/cudaerror.hpp:6-18).  Here each becomes a return code. */
typedef enum {
  MPX_OK = 0,
  MPX_ERR_INVALID = 1,     /* bad argument               (std::invalid_argument) */
  MPX_ERR_RANGE = 2,       /* index / grid out of range  (std::out_of_range)     */
  MPX_ERR_RUNTIME = 3,     /* invalid state              (std::runtime_error)    */
  MPX_ERR_NOMEM = 4,       /* device memory exhausted or over the engine budget  */
  MPX_ERR_CUDA = 5,        /* CUDA runtime error                                 */
  MPX_ERR_UNSUPPORTED = 6, /* configuration outside what the kernels implement   */
  MPX_ERR_TIMEOUT = 7,     /* bounded wait expired                               */
  MPX_ERR_NODEVICE = 8     /* no CUDA device                                     */
} mpx_status;

/* Quantities for mpx_eval / mpx_average / mpx_energy.  Names follow the
 * reference's Ferromagnet properties (mumaxplus/ferromagnet.py:678-901). */
typedef enum {
  MPX_Q_MAGNETIZATION = 0,
  MPX_Q_EFFECTIVE_FIELD = 1,    /* physics/effectivefield.cpp:15-28 */
  MPX_Q_EXCHANGE_FIELD = 2,     /* physics/exchange.cu:204-239      */
  MPX_Q_DMI_FIELD = 3,          /* physics/dmi.cu:242-269           */
  MPX_Q_ANISOTROPY_FIELD = 4,   /* physics/anisotropy.cu:109-140    */
  MPX_Q_EXTERNAL_FIELD = 5,     /* physics/zeeman.cu:53-91          */
  MPX_Q_DEMAG_FIELD = 6,        /* physics/demag.cpp:13-19          */
  MPX_Q_TORQUE = 7,             /* physics/torque.cu:14-19          */
  MPX_Q_LLG_TORQUE = 8,         /* physics/torque.cu:47-56          */
  MPX_Q_DAMPING_TORQUE = 9,     /* physics/torque.cu:58-87          */
  /* scalar (1-component) energy densities, J/m^3 (physics/energy.cu:18-50) */
  MPX_Q_EXCHANGE_ENERGY_DENSITY = 10,
  MPX_Q_DMI_ENERGY_DENSITY = 11,
  MPX_Q_ANISOTROPY_ENERGY_DENSITY = 12,
  MPX_Q_ZEEMAN_ENERGY_DENSITY = 13,
  MPX_Q_DEMAG_ENERGY_DENSITY = 14,
  MPX_Q_TOTAL_ENERGY_DENSITY = 15,
  MPX_Q_SPIN_TRANSFER_TORQUE = 16,   /* physics/stt.cu:143-185 (Zhang-Li or Slonczewski), 1/s */
  MPX_Q_COUNT = 17
} mpx_quantity;
/* energy densities are the scalar quantities; the others have 3 components */
#define MPX_Q_IS_SCALAR(q) ((q) >= MPX_Q_EXCHANGE_ENERGY_DENSITY && (q) <= MPX_Q_TOTAL_ENERGY_DENSITY)

/* Runge-Kutta methods (core/butchertableau.cpp). */
typedef enum {
  MPX_RK_HEUN = 0,
  MPX_RK_BOGACKI_SHAMPINE = 1,
  MPX_RK_CASH_KARP = 2,
  MPX_RK_FEHLBERG = 3,       /* reference default (core/timesolver.cpp:17-19) */
  MPX_RK_DORMAND_PRINCE = 4
} mpx_rk_method;

typedef struct mpx_engine mpx_engine;

/* A material parameter: a uniform value, or per-cell values (host pointer,
 * ncells floats; NULL means uniform).  core/parameter.hpp:16-110. */
typedef struct {
  double uniform;
  const float* cells;
} mpx_scalar;

/* A vector parameter: uniform value or per-cell SoA values (3*ncells floats).
 * core/parameter.hpp:115-240. */
typedef struct {
  double uniform[3];
  const float* cells;
} mpx_vector;

/* Order of the DMI tensor components in mpx_magnet_desc.dmi
 * (physics/dmitensor.hpp; interfacial DMI sets xxz = yyz = D). */
enum {
  MPX_DMI_XXY = 0, MPX_DMI_XXZ, MPX_DMI_XYZ,
  MPX_DMI_YXY, MPX_DMI_YXZ, MPX_DMI_YYZ,
  MPX_DMI_ZXY, MPX_DMI_ZXZ, MPX_DMI_ZYZ
};

/* One ferromagnet.  Geometry/regions/mastergrid/PBC follow core/system.hpp:10-119,
 * core/grid.hpp:7-89 and core/world.hpp.  All pointers are host pointers, read
 * during the call only. */
typedef struct {
  int size[3];                  /* nx, ny, nz                                   */
  int origin[3];                /* grid origin in cells                         */
  double cellsize[3];           /* m                                            */
  int mastergrid_size[3];       /* periodic box; 0 = not periodic on that axis  */
  int mastergrid_origin[3];
  int pbc_repetitions[3];       /* image range of the demag kernel              */
  const unsigned char* geometry;  /* ncells bytes (1 = in geometry) or NULL     */
  const unsigned int* regions;    /* ncells region indices or NULL (all 0)      */
  mpx_scalar msat;              /* A/m   (reference default 1)                  */
  mpx_scalar aex;               /* J/m   (default 0)                            */
  mpx_scalar alpha;             /* (default 0)                                  */
  mpx_scalar ku1, ku2;          /* J/m^3 (default 0)                            */
  mpx_scalar frozen_spins;      /* nonzero = frozen (default 0)                 */
  mpx_vector anis_u;            /* uniaxial axis, normalised per cell           */
  mpx_vector bias_magnetic_field; /* per-magnet bias, T                         */
  mpx_scalar dmi[9];            /* J/m^2, order MPX_DMI_*                       */
  int lut_regions;              /* region count covered by the two LUTs below   */
  double inter_exchange;        /* uniform inter-region exchange (default 0)    */
  const float* inter_exchange_lut;  /* lut_regions*(lut_regions-1)/2 or NULL    */
  double scale_exchange;        /* uniform inter-region scale (default 1)       */
  const float* scale_exchange_lut;
  int enable_demag;             /* default 1                                    */
  int enable_openbc;            /* default 0                                    */
  /* cubic anisotropy (physics/anisotropy.cu:57-106); used when the uniaxial
   * term is assured zero, as in the reference */
  mpx_scalar kc1, kc2, kc3;     /* J/m^3                                        */
  mpx_vector anis_c1, anis_c2;  /* cubic axes (normalised per cell; c3 = c1 x c2) */
  /* stray fields between the magnets of one group (physics/zeeman.cu:70-88):
   * Magnet::enableAsStrayFieldSource / Destination, inverted so that the
   * zero default keeps both on */
  int stray_source_off;
  int stray_destination_off;
  /* spin-transfer torque (physics/stt.cu; physics/ferromagnet.cpp:34-52 defaults) */
  mpx_scalar pol, xi, lambda, epsilon_prime;
  mpx_scalar free_layer_thickness;  /* m; the reference's default is nz * cellsize z */
  mpx_vector jcur;                  /* A/m^2 */
  mpx_vector fixed_layer;           /* Slonczewski polarisation direction p */
  int fixed_layer_below;            /* 0: fixed layer on top (reference default) */
  int zhang_li_off;                 /* enableZhangLiTorque, inverted */
  int slonczewski_off;              /* enableSlonczewskiTorque, inverted */
  /* thermal noise (physics/thermalnoise.cu): temperature in K and the seed of
   * the counter-based generator (the reference seeds cuRAND with the clock) */
  mpx_scalar temperature;
  uint64_t thermal_seed;
} mpx_magnet_desc;

/* Time-solver settings (core/timesolver.hpp:74-82 defaults in brackets). */
typedef struct {
  int method;                       /* mpx_rk_method [FEHLBERG]        */
  int adaptive;                     /* [1]                             */
  double max_error;                 /* [1e-5]                          */
  double headroom;                  /* [0.8]                           */
  double lower_bound;               /* [0.5]                           */
  double upper_bound;               /* [2.0]                           */
  double sensible_factor;           /* [0.01]                          */
  double sensible_timestep_default; /* [1e-14]                         */
} mpx_solver_params;

/* Per-group counters and state. */
typedef struct {
  double time, timestep;
  int64_t steps, rejected, evaluations;
  int status;            /* 0 idle, 1 running, 2 finished, 3 failed (NaN) */
  double last_error;     /* last max-norm error estimate                  */
  double max_torque;     /* max |torque| at the last check (rad/s), or -1 */
} mpx_group_info;

/* ---- library ---------------------------------------------------------- */
const char* mpx_version(void);
/* Message of the last failing call on this thread ("" if none). */
const char* mpx_last_error(void);
/* Number of CUDA devices visible (0 if none). */
int mpx_device_count(void);

/* ---- engine (one GPU, one stream) -------------------------------------- */
mpx_status mpx_engine_create(int device, mpx_engine** out);
mpx_status mpx_engine_destroy(mpx_engine* e);
/* Launch subsequent work on this cudaStream_t (NULL = the engine's own stream). */
mpx_status mpx_engine_set_stream(mpx_engine* e, void* stream);
mpx_status mpx_engine_synchronize(mpx_engine* e);
/* Arithmetic of the y transforms of the demag convolution (the cuFFT y
 * stages of physics/strayfieldfft.cu:216-218, 238-240).  MPX_DFT_FP32
 * (default): shared-memory FFTs in FP32 on the CUDA cores.  MPX_DFT_TF32X3:
 * for y lengths 1024 and 2048, the 32-point DFT stages as TF32 tensor-core
 * GEMMs (tcgen05) with 3xTF32 split products accumulated in FP32, in the
 * three-pass y / z / y form; other lengths keep the FP32 FFTs.  Applies to
 * the magnets added afterwards: set it before the first mpx_magnet_add
 * (MPX_ERR_INVALID otherwise). */
enum { MPX_DFT_FP32 = 0, MPX_DFT_TF32X3 = 1 };
mpx_status mpx_engine_set_dft(mpx_engine* e, int mode);
/* Number of waits of the tensor-core kernels on their MMA completion that
 * gave up (each bounded at about 0.3 s; the kernel then stops its work and
 * releases its tensor memory instead of hanging), since the last call, on the
 * current device; synchronises the device and clears the count. */
mpx_status mpx_tc_status(unsigned int* timeouts);
/* No counterpart in the reference.  Exercises the timeout path of the
 * tensor-core kernels without a fault: one block on the current device takes
 * tensor memory and waits (at most about 1 ms) on an mbarrier that nothing
 * arrives at, then counts the timeout, releases its tensor memory and returns.
 * *timeouts: the count read back (1 expected); the device stays usable. */
mpx_status mpx_tc_timeout_selftest(unsigned int* timeouts);
/* Uniform field over the whole world, T (physics/mumaxworld.hpp biasMagneticField). */
mpx_status mpx_engine_set_world_bias(mpx_engine* e, const double b[3]);
/* Device bytes currently held by the engine (buffers, spectra, kernels). */
mpx_status mpx_engine_memory(mpx_engine* e, int64_t* bytes);
/* Number of kernels this engine has launched since creation. */
mpx_status mpx_engine_launch_count(mpx_engine* e, int64_t* count);
/* No counterpart in the reference.  How often the CUDA graphs of one attempt
 * were instantiated anew and how often an existing one was updated in place
 * (a solve that starts or finishes changes only the launch sizes and tables,
 * so the graph is updated rather than rebuilt). */
mpx_status mpx_engine_graph_stats(mpx_engine* e, int64_t* instantiations, int64_t* updates);

/* ---- solve groups: magnets that share one time and time step ----------- */
mpx_status mpx_group_create(mpx_engine* e, int* group);
mpx_status mpx_group_destroy(mpx_engine* e, int group);   /* removes its magnets */
mpx_status mpx_group_info_get(mpx_engine* e, int group, mpx_group_info* out);
/* Checkpoint / resume of a group (no counterpart in the reference, whose state
 * is reachable only through magnetization.get/set and time/timestep).  The
 * snapshot holds the time, time step, accepted-step count (the counter of the
 * thermal noise generator), whether the FSAL derivative k0 is valid, and per
 * magnet of the group (in the order added) its state m and k0, 3 * ncells floats
 * each, copied without normalisation.  Loading a snapshot into a group of
 * magnets of the same sizes continues exactly as the saved run would have.
 * A group that is running (started by mpx_group_start and not yet finished)
 * is refused with MPX_ERR_INVALID; loading clears the final-step state of an
 * earlier run.  mpx_group_state_bytes gives the size of the host buffer. */
mpx_status mpx_group_state_bytes(mpx_engine* e, int group, int64_t* bytes);
mpx_status mpx_group_save(mpx_engine* e, int group, void* buf, int64_t bytes);
mpx_status mpx_group_load(mpx_engine* e, int group, const void* buf, int64_t bytes);

/* ---- magnets ------------------------------------------------------------ */
/* Adds a ferromagnet to `group`; builds its FP64 Newell kernel spectrum when
 * demag is enabled.  The initial magnetization is random unit vectors seeded by
 * the magnet id (the reference seeds with the clock, ferromagnet.cpp:62-76);
 * an adaptive group's time step becomes the sensible one for that state
 * (core/timesolver.cpp:49-52). */
mpx_status mpx_magnet_add(mpx_engine* e, int group, const mpx_magnet_desc* d, int* magnet);
/* mpx_magnet_add with the initial magnetization given (3 * ncells floats, SoA,
 * host memory unless on_device; normalised as by mpx_magnet_set_m) instead of
 * the random one: one field evaluation (the sensible time step of an adaptive
 * group, for this state) instead of two, no separate set_m.  No counterpart in
 * the reference, where a new magnet starts random and is then set. */
mpx_status mpx_magnet_add_state(mpx_engine* e, int group, const mpx_magnet_desc* d, const float* m0, int on_device,
                                int* magnet);
/* Device bytes mpx_magnet_add would take for `d`: *resident stays allocated
 * until the magnet is removed (state buffers, spectra, per-cell parameters,
 * work tables); *transient is the extra peak while it is added (the FP64
 * kernel construction buffers).  No engine or device needed; used to admit
 * solves against a memory budget.  No counterpart in the reference, which
 * allocates from its pool as fields are needed (core/gpumemorypool.cu). */
mpx_status mpx_magnet_bytes(const mpx_magnet_desc* d, int64_t* resident, int64_t* transient);
/* Re-reads all parameters; rebuilds the demag kernel only when the cell size,
 * geometry-independent grid data, mastergrid or PBC changed. */
mpx_status mpx_magnet_update(mpx_engine* e, int magnet, const mpx_magnet_desc* d);
mpx_status mpx_magnet_remove(mpx_engine* e, int magnet);
/* Sets m (3*N floats) and normalises it per cell (core/variable.cpp:76-87). */
mpx_status mpx_magnet_set_m(mpx_engine* e, int magnet, const float* m, int on_device);
mpx_status mpx_magnet_get_m(mpx_engine* e, int magnet, float* m, int on_device);
/* Evaluates a quantity into out (3*N floats, or N for energy densities).
 * on_device: 0 = out is a host pointer, 1 = out is a device pointer,
 * 2 = evaluate into the engine's scratch buffer only (out may be NULL). */
mpx_status mpx_eval(mpx_engine* e, int magnet, int quantity, float* out, int on_device);
/* Per-component mean over the cells in the geometry, FP64 accumulation
 * (core/reduce.cu:101-151). */
mpx_status mpx_average(mpx_engine* e, int magnet, int quantity, double out[3]);
/* Max |v| over the geometry (core/reduce.cu:53-99), FP64 accumulation. */
mpx_status mpx_max_norm(mpx_engine* e, int magnet, int quantity, double* out);
/* Energy of a term = ncells * <energy density> * cell volume (physics/energy.cu:52-92). */
mpx_status mpx_energy(mpx_engine* e, int magnet, int quantity, double* out);
/* Measurement: times each kernel of one effective-field evaluation of `magnet`
 * with CUDA events on the engine's stream, `reps` times after one warm-up, and
 * writes the mean milliseconds per launch of [x-forward FFT, y/z FFT + kernel
 * multiply, x-inverse FFT + epilogue, local-terms-only] (0 for kernels the
 * magnet does not use).  No reference counterpart (FieldQuantity::_bench times
 * the whole evaluation, mumaxplus/fieldquantity.py:111-118). */
mpx_status mpx_profile_eval(mpx_engine* e, int magnet, int reps, double ms[4]);
/* Measurement of the batched launches: times, with CUDA events, the kernels of
 * stage 1 of one Runge-Kutta attempt over every started group (the launch
 * tables of mpx_advance), `reps` times after one warm-up, without the step
 * controller, and writes the mean milliseconds of [stage combination + x-forward
 * (or k_combine), stray-field pairs, y/z passes (all z classes and the split
 * path), x-inverse + epilogue (or k_local)].  Stage 1 only writes the stage
 * state and k_1, which the next attempt recomputes; the solves do not advance.
 * Needs the method the groups run with.  No reference counterpart. */
mpx_status mpx_profile_attempt(mpx_engine* e, int method, int reps, double ms[4]);
/* Shape autotuner for the started groups: times stage 1 of an attempt (as
 * mpx_profile_attempt) with the default row-tile and y/z-block shapes divided by
 * 1, 2, 4 and 8 (then the two-blocks-per-SM rule), and keeps the fastest divisor
 * for the x passes and for the y/z passes while the started magnets keep more
 * than half of the cells they had at tuning.  Call after one mpx_advance (k0 of the started solves valid).  The
 * divisors chosen go to *div_x, *div_yz.  No reference counterpart. */
mpx_status mpx_autotune(mpx_engine* e, int method, int* div_x, int* div_yz);
/* Real-space demag kernel, 6*K floats on the reference's kernel grid
 * (physics/strayfieldkernel.cu:80-99; bindings/wrap_magnet.cpp:56-59).
 * dims receives the kernel grid size (Kx, Ky, Kz). Pass out=NULL to query dims. */
mpx_status mpx_demag_kernel(mpx_engine* e, int magnet, float* out, int dims[3]);
/* Stray field (T) of magnet `src`'s current state on a destination grid:
 * StrayField(magnet, grid).eval() (physics/strayfield.cpp:45-82,
 * bindings/wrap_strayfield.cpp:12-24) when dst_magnet < 0 -- the grid of
 * `size` cells at `origin` (cell units, the source's cell size), every cell --
 * or Magnet.stray_field_from_magnet(source).eval() (bindings/wrap_magnet.cpp:
 * 45-52) when dst_magnet >= 0 -- that magnet's grid, zero outside its
 * geometry; both magnets must belong to one group (world), else
 * MPX_ERR_RUNTIME.  method MPX_STRAY_FFT (the reference's default: FFT
 * convolution on the pair's kernel grid, n_src + n_dst - 1 cells per axis,
 * physics/strayfieldkernel.cu:80-99; the direct sum where a padded length
 * would exceed 4096 along x or y or 2048 along z) or
 * MPX_STRAY_BRUTE (direct sum over the source cells,
 * physics/strayfieldbrute.cu:15-57); both include the world's periodic images
 * (the source's mastergrid and repetitions).  out: 3 x ncells floats (SoA),
 * host memory unless on_device. */
enum { MPX_STRAY_FFT = 0, MPX_STRAY_BRUTE = 1 };
mpx_status mpx_stray_field(mpx_engine* e, int src, int dst_magnet, const int size[3], const int origin[3], int method,
                           float* out, int on_device);

/* ---- time solver of a group (core/timesolver.cpp) ----------------------- */
mpx_status mpx_solver_set_params(mpx_engine* e, int group, const mpx_solver_params* p);
mpx_status mpx_solver_get_params(mpx_engine* e, int group, mpx_solver_params* p);
mpx_status mpx_solver_set_time(mpx_engine* e, int group, double t);
mpx_status mpx_solver_get_time(mpx_engine* e, int group, double* t);
mpx_status mpx_solver_set_timestep(mpx_engine* e, int group, double dt);
mpx_status mpx_solver_get_timestep(mpx_engine* e, int group, double* dt);
/* sensibleFactor / max|torque| (core/timesolver.cpp:37-47). */
mpx_status mpx_solver_sensible_timestep(mpx_engine* e, int group, double* dt);
/* TimeSolver::step / steps / run (core/timesolver.cpp:77-111).  Blocking. */
mpx_status mpx_solver_step(mpx_engine* e, int group);
mpx_status mpx_solver_steps(mpx_engine* e, int group, int nsteps);
mpx_status mpx_solver_run(mpx_engine* e, int group, double duration);
/* The loop of TimeSolver.solve (mumaxplus/timesolver.py:114-152) for average
 * magnetizations, without a host round trip per time point: for k = 0..n-1,
 * run(times[k] - t), then record row k of `out` (n rows of 1 + 3 * nmag doubles:
 * the time, then <m> of every magnet of the group in the order they were added,
 * each exactly as mpx_average of MPX_Q_MAGNETIZATION would give it).  The time
 * points, the run() logic between them and the averages stay on the device;
 * the table comes back once at the end.  times must be non-decreasing
 * (MPX_ERR_INVALID otherwise).  Blocking. */
mpx_status mpx_solver_run_sampled(mpx_engine* e, int group, const double* times, int n, double* out);

/* Minimizer::exec (physics/minimizer.cu:73-160): steepest descent on the
 * damping torque with Barzilai-Borwein step sizes over the group's magnets,
 * until the last nsamples x (number of magnets) largest per-cell changes of m
 * are all <= tol.  The time and time step are left as they were. */
mpx_status mpx_minimize(mpx_engine* e, int group, double tol, int nsamples);
/* Relaxer::exec (physics/relaxer.cpp:88-174): adaptive Fehlberg steps of the
 * damping torque (no precession) while the total energy decreases, then, with a
 * negative threshold, lowering the maximum error by sqrt(2) down to tol while the
 * summed squared torque decreases; with a positive threshold, lowering it each time
 * every magnet's maximum torque is at or below the threshold.  Restores the solver
 * settings, time and time step afterwards (an adaptive solver then takes the
 * sensible time step).  threshold == 0 is MPX_ERR_INVALID. */
mpx_status mpx_relax(mpx_engine* e, int group, double tol, double threshold);

/* ---- many groups at once (batched / served forms) ----------------------- */
/* Arms `group` to run for `duration` seconds, or until max|torque|/gamma_LL
 * drops below torque_stop tesla (torque_stop <= 0 disables that test).  The
 * group then advances with every mpx_advance call until it finishes. */
mpx_status mpx_group_start(mpx_engine* e, int group, double duration, double torque_stop);
/* Enqueues `attempts` Runge-Kutta attempts for every armed group (asynchronous,
 * CUDA-graph replay).  Only the magnets of started groups are in the launch
 * tables; a group that finishes on the device skips its work until the next
 * mpx_poll takes it out of the tables. */
mpx_status mpx_advance(mpx_engine* e, int attempts);
/* Waits for enqueued work; writes up to `cap` ids of groups that finished
 * since the last poll into done[] and their count into *n_done, and the number
 * of groups still running into *n_running. */
mpx_status mpx_poll(mpx_engine* e, int* done, int cap, int* n_done, int* n_running);

/* ---- allocation-free reduction ------------------------------------------ */
/* No counterpart in the reference.  For callers that may not allocate device
 * memory (a monitoring hook inside another application's loop, held to a fixed
 * device-memory budget, that must not add a cudaMalloc's synchronisation or
 * out-of-memory failure).  Reduces a field the caller holds on the current
 * device -- `field` is SoA, ncomp components of `ncells` floats, `geometry`
 * optional (NULL = all cells) -- over the cells in the geometry: op 0 =
 * per-component sum, op 1 = max |v| (in out[0]); FP64 accumulation, the same
 * kernels as mpx_average / mpx_max_norm.  Allocates nothing: its scratch is a
 * static device array of 6168 bytes (256 block partials x 3 + 3 results) that
 * every GPU loading the library holds until exit.  ncells must be in
 * [1, 715827882] and ncomp in [1, 3]; larger sizes are rejected with
 * MPX_ERR_INVALID.  The first call on a device looks up the array's device
 * address (set-up); make that first call before any stream capture.  The
 * address stays cached for the life of the process: do not use the library
 * across a cudaDeviceReset of that device.  All calls share the array: calls
 * that overlap on the GPU race.  A CUDA error already pending on the calling
 * thread is returned as MPX_ERR_CUDA and left pending (not cleared).  Blocks
 * until `out` is written; `stream` NULL = the legacy default stream. */
mpx_status mpx_reduce_noalloc(const float* field, int ncells, int ncomp, const unsigned char* geometry, int op,
                              void* stream, double out[3]);

/* No counterpart in the reference (it has no sanitizer or checked build):
 * index checking for the checked library libmpx_checked.so, built from the
 * same sources with -DMPX_BOUNDS_CHECK.  There every per-cell access of a
 * field buffer (stencil neighbours, stage states and derivatives, stray-field
 * buffers) verifies 0 <= i < N; a bad access is skipped (loads give 0) and the
 * first one recorded, without trapping.  Synchronises the current device,
 * writes the record to *first_bad (0 = none; else bit 63 set, N in bits
 * 32..62, i in bits 0..31) and clears it.  The four-cell vector accesses of
 * the forward x pass, the spectrum stores / gathers of the x passes, and in
 * the y/z passes the spectrum column gathers and scatters, the kernel-spectrum
 * reads and the split path's y-transformed spectrum (FFT and tensor-core
 * forms), and the stray-field FFT passes on the pair grid (tables, work and
 * kernel spectra, destination cells) are checked the same way.  In libmpx.so
 * the checks are compiled out
 * and this returns MPX_ERR_UNSUPPORTED. */
mpx_status mpx_bounds_check(unsigned long long* first_bad);

#ifdef __cplusplus
}
#endif
#endif /* MPX_H */
