/* adaptflood.h -- C ABI of the B200-native AdaptFlood local-inertial time step.
 *
 * Three layers share this header (plus the input-file reader):
 *
 * 1. The drop-in layer (af_update_qs ... af_fill).  One entry point per
 *    function of the reference's src/kernels.hpp plus the three pieces of
 *    device work that src/main.cpp does inline.  Arguments keep the
 *    reference's names, order and meaning; arrays are DEVICE pointers in the
 *    reference's layout:
 *        cells  c(i,j) = i + j*xsz                 xsz*ysz entries
 *        faces  f(i,j) = i + j*(xsz+1)             (xsz+1)*(ysz+1) entries
 *    (Qx(i,j) = west face of cell (i,j), Qy(i,j) = north face; row 0 north.)
 *    Every call enqueues on `stream` (a cudaStream_t; NULL = legacy default
 *    stream) and waits for it before returning, as each reference function
 *    ends in Kokkos::fence().  The reference's functions return void and abort
 *    on error; these return AF_OK or a negative AF_E* code.
 *
 * 2. The simulation layer (af_sim_*): one fused, graph-launched kernel per
 *    time step with device-resident dt, time and hydrograph interpolation, in
 *    FP64 (results within 1e-9 m of the reference) or FP32 state with FP64
 *    time, interpolation and volume accumulation.
 *
 * 3. The batch layer (af_batch_*): many grids of uneven sizes with their own
 *    dt stepped together by one persistent, graph-launched kernel, placed in
 *    one device arena and admitted by memory footprint (continuous batching).
 *
 * Point boundaries: the reference's src/main.cpp:256-260 scatter and
 * src/kernels.cpp:261-274 overwrite run one thread per boundary and race when
 * two boundaries share a cell.  Here both are deterministic and equal to the
 * sequential file-order result: sources on one cell accumulate in file order,
 * and of several depth BCs on one cell the last in file order wins.
 */
#ifndef ADAPTFLOOD_H
#define ADAPTFLOOD_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ----------------------------------------------------------------- errors */
#define AF_OK 0
#define AF_EINVAL (-1)  /* null pointer, negative size, unsupported shape      */
#define AF_ERANGE (-2)  /* grid beyond int32 indexing, or an index off the grid */
#define AF_ECUDA (-3)   /* CUDA runtime error (see af_last_cuda_error)         */
#define AF_ENOMEM (-4)  /* device or host allocation failed                     */
#define AF_EIO (-5)     /* an input file is missing or malformed                */
#define AF_ESTATE (-6)  /* the device reported a bad state (e.g. step overflow) */

const char* af_strerror(int code);
/* The last CUDA error string seen by this library on the calling thread. */
const char* af_last_cuda_error(void);
int af_version(void);

/* Boundary types (src/types.hpp:41-48) and the device point-BC codes
 * (src/main.cpp:187-189). */
enum { AF_BC_CLOSED = 0, AF_BC_FREE = 1, AF_BC_HFIX = 2, AF_BC_HVAR = 3,
       AF_BC_QFIX = 4, AF_BC_QVAR = 5 };

/* ===================================================== 1. drop-in layer == */

/* Replaces UpdateQs_GPU (src/kernels.hpp:8-9, src/kernels.cpp:6-19):
 * Qxold = Qx*(1/dx), Qyold = Qy*(1/dx) over all (xsz+1)*(ysz+1) faces. */
int af_update_qs(const double* Qx, const double* Qy, double* Qxold, double* Qyold, int xsz,
                 int ysz, double dx, void* stream);

/* Replaces FloodplainQ_GPU (src/kernels.hpp:12-16, src/kernels.cpp:22-146):
 * Hmax over valid cells -> *Tstep = cfl*dx/sqrt(g*Hmax) (or InitTstep when
 * Hmax <= DepthThresh), then the interior x- and y-face fluxes.  *Tstep is a
 * HOST pointer, written before return.  dy, dhlin, Qlimfact and dA are
 * accepted and unused, as in the reference. */
int af_floodplain_q(const double* H, const double* DEM, double* Qx, double* Qy,
                    const double* Qxold, const double* Qyold, int xsz, int ysz, double dx,
                    double dy, double FPn, double DepthThresh, double MaxHflow, double dhlin,
                    double* Tstep, double Qlimfact, double dA, double cfl, double g,
                    double InitTstep, double theta, double nodata, void* stream);

/* Replaces BCs_GPU (src/kernels.hpp:19-21, src/kernels.cpp:149-256): edge
 * faces, FREE outflow or CLOSED (0).  dt is accepted and unused.  A grid one
 * column wide with west_free set is rejected (AF_EINVAL): the reference reads
 * past the grid there. */
int af_bcs(double* Qx, double* Qy, const double* H, const double* DEM, int xsz, int ysz,
           double dx, double g, double dt, double nodata, int west_free, int east_free,
           int north_free, int south_free, void* stream);

/* Replaces ApplyPointBCs_GPU (src/kernels.hpp:24-25, src/kernels.cpp:259-277):
 * type 1 (FREE) sets H = 0, types 2/3 (HFIX/HVAR) set H = value; other types
 * do nothing.  An index outside [0, ncells) is skipped and the call returns
 * AF_ERANGE.  ncols, dx, dA, Tstep are accepted and unused, as in the
 * reference; ncells is the grid's cell count (added for the bounds check). */
int af_apply_point_bcs(double* H, const int* bc_idx, const int* bc_type, const double* bc_value,
                       int num_bcs, int ncols, double dx, double dA, double Tstep, int ncells,
                       void* stream);

/* Replaces UpdateH_GPU (src/kernels.hpp:28, src/kernels.cpp:280-290). */
int af_update_h(double* H, const double* Qx, const double* Qy, int xsz, int ysz, double dA,
                double Tstep, void* stream);

/* Replaces ComputeVelocity_GPU (src/kernels.hpp:31-33, src/kernels.cpp:293-351). */
int af_compute_velocity(double* Vx, double* Vy, const double* H, const double* DEM,
                        const double* Qx, const double* Qy, int xsz, int ysz, double dx,
                        double nodata, void* stream);

/* Replaces Rainfall_GPU (src/kernels.hpp:36-37, src/kernels.cpp:354-367). */
int af_rainfall(double* H, const double* DEM, int xsz, int ysz, double rain_rate, double Tstep,
                double nodata, void* stream);

/* Replaces the inline AddFlowBCs scatter of src/main.cpp:256-260:
 * H(idx) = max(H(idx) + ps_flow, 0) per source, where the caller forms
 * ps_flow = q*dx*Tstep/dA as src/main.cpp:253 does.  Indices outside
 * [0, ncells) are skipped and the call returns AF_ERANGE. */
int af_add_point_sources(double* H, const int* ps_idx, const double* ps_flow, int num,
                         int ncells, void* stream);

/* No counterpart in the reference.  The same scatter as af_add_point_sources,
 * for callers that cannot let this library allocate device memory: a host
 * application that hands all device memory to its own pool or arena (so a
 * library cudaMalloc would fail or fragment it), or one that cannot afford
 * the device-wide synchronisation a cudaFree implies.  It calls no
 * cudaMalloc, cudaFree or other allocating routine; its sort keys live in a
 * fixed device array compiled into the library (about 33 KB on every GPU
 * that loads it, held until the process exits).
 *   - num may be at most AF_NOALLOC_MAX_SOURCES; a larger num returns
 *     AF_ERANGE before anything runs, and H is left unchanged.  Indices off
 *     the grid are skipped and reported with AF_ERANGE, as in
 *     af_add_point_sources.
 *   - Each call looks up the array's device address on the current device
 *     (the first call on a device loads the library's device code there),
 *     then waits for `stream` before it returns (it reads an error flag back
 *     to the host): the call is synchronous, and it must not be made while
 *     `stream` is being captured into a graph.
 *   - Every call shares the one array: calls whose work overlaps on the GPU
 *     (concurrent streams or host threads) race and must be serialised by
 *     the caller.  Each call clears the state it relies on. */
#define AF_NOALLOC_MAX_SOURCES 4096
int af_add_point_sources_noalloc(double* H, const int* ps_idx, const double* ps_flow, int num,
                                 int ncells, void* stream);

/* Replaces the inline Vol/Area reductions of src/main.cpp:293-298:
 * *vol = sum H*dA, *area = sum of dA over H > 0.01 (HOST outputs).  The sum
 * is formed in a fixed order, so repeated calls agree bit for bit. */
int af_volume_area(const double* H, int64_t n, double dA, double* vol, double* area,
                   void* stream);

/* Replaces the inline Init* fills of src/main.cpp:156-160. */
int af_fill(double* x, int64_t n, double value, void* stream);

/* No counterpart in the reference's interface: evaluates, over a device
 * array, the pow that the FP64 kernels use for the friction term's
 * pow(hflow, 10.0/3.0) (src/kernels.cpp:83,133): out[k] = x[k]^y.  It is the
 * C library's (glibc >= 2.28) table-driven algorithm restated, and returns
 * glibc's value on all but about 1e-7 of positive normal arguments; a caller
 * can compare it with its own C library here.  Synchronous on `stream`. */
int af_pow_eval(const double* x, double* out, int64_t n, double y, void* stream);

/* ================================================== 2. simulation layer == */

enum { AF_PREC_F64 = 0, AF_PREC_F32 = 1 };

/* Grid and scalar parameters of one case (src/main.cpp:115-124). */
typedef struct af_case_desc {
  int nx, ny;            /* ncols, nrows                                     */
  double dx;             /* cellsize; dy = dx and dA = dx*dx as in the reference */
  double nodata;         /* DEM nodata value                                  */
  double fpn;            /* Manning n (par key fpfric)                        */
  double depth_thresh;   /* par key depth_thresh                              */
  double cfl;            /* par key cfl                                       */
  double init_tstep;     /* par key initial_tstep                             */
  double g;              /* 9.81 in the reference                             */
  double max_hflow;      /* 10.0 in the reference                             */
  double theta;          /* 1.0 in the reference                              */
  int west_free, east_free, north_free, south_free;
  double mass_int;       /* volume/area report interval (s); <= 0: never      */
} af_case_desc;

/* Point boundaries and rain, HOST arrays (copied at create time).  Flow
 * sources keep file order with type AF_BC_QFIX/AF_BC_QVAR; other point BCs
 * keep file order with device codes 1/2/3 (FREE/HFIX/HVAR).  Hydrographs are
 * CSR: entries off[k]..off[k+1] of times/vals; an empty series means the
 * fixed value (src/io.cpp:300).  Rain: n_rain == 0 disables rainfall. */
typedef struct af_forcing_desc {
  int n_flow;
  const int* flow_idx;
  const int* flow_type;
  const double* flow_value;
  const int* flow_off;
  const double* flow_times;
  const double* flow_vals;
  int n_other;
  const int* other_idx;
  const int* other_type;
  const double* other_value;
  const int* other_off;
  const double* other_times;
  const double* other_vals;
  int n_rain;
  const double* rain_times;
  const double* rain_rates;
} af_forcing_desc;

typedef struct af_sim af_sim;

/* Creates a device-resident simulation on `device` from HOST arrays: dem
 * (nx*ny, reference layout) and optional initial depth h0 (NULL = zeros, as
 * src/main.cpp:156).  precision is AF_PREC_F64 or AF_PREC_F32. */
int af_sim_create(const af_case_desc* c, const af_forcing_desc* f, const double* dem,
                  const double* h0, int precision, int device, af_sim** out);
int af_sim_destroy(af_sim* s);

/* Enqueues steps while t < t_stop and fewer than max_steps steps have run in
 * this call (the loop test of src/main.cpp:227), without waiting. */
int af_sim_launch(af_sim* s, double t_stop, int64_t max_steps);
/* Waits for the enqueued steps. */
int af_sim_sync(af_sim* s);
/* af_sim_launch + af_sim_sync; *steps_done (optional) gets the step count. */
int af_sim_run(af_sim* s, double t_stop, int64_t max_steps, int64_t* steps_done);
/* Time, last dt, current Hmax and total steps (after a sync). */
int af_sim_status(af_sim* s, double* t, double* dt_last, double* hmax, int64_t* steps);
/* The device stream the simulation runs on (a cudaStream_t). */
void* af_sim_stream(af_sim* s);

/* State in the reference layout, HOST arrays, FP64: H (nx*ny), Qx and Qy
 * ((nx+1)*(ny+1), including the never-written corner slots as 0).  Any
 * pointer may be NULL. */
int af_sim_get_state(af_sim* s, double* H, double* Qx, double* Qy);
int af_sim_set_state(af_sim* s, const double* H, const double* Qx, const double* Qy, double t);
/* Velocity of the current state (ComputeVelocity_GPU semantics), HOST. */
int af_sim_velocity(af_sim* s, double* Vx, double* Vy);
/* Volume and flooded area of the current state (FP64 accumulation). */
int af_sim_volume(af_sim* s, double* vol, double* area);
/* The mass-report series recorded at each mass_int crossing
 * (src/main.cpp:291-304): up to cap entries of (t, vol, area). */
int af_sim_mass_series(af_sim* s, double* t, double* vol, double* area, int cap, int* n);

/* Checkpoint and restart (no counterpart in the reference, which always starts
 * at t = 0): af_sim_checkpoint writes the whole simulation state (fields in the
 * state precision, time, step count, dt inputs, rain rate, mass-report series)
 * to a binary file; af_sim_restore loads it into a simulation created from the
 * same case and precision (AF_EINVAL otherwise), after which the run continues
 * bit for bit as if it had never stopped.  Files use the host's byte order. */
int af_sim_checkpoint(af_sim* s, const char* path);
int af_sim_restore(af_sim* s, const char* path);

/* Output of a run as the reference's main loop writes it (src/main.cpp:196-388,
 * src/io.cpp:314-334, src/async_output.cpp:84-176): ESRI ASCII grids with
 * "%.4f " values in out_dir (created if missing): H_0000.asc for the state at
 * the start, H_%04d.asc after the first step ending at or past each multiple
 * of save_int (with Vx_/Vy_%04d.asc too when voutput and async_style, as the
 * reference's async writer does), stage.csv rows ("%.1f" time, ",%.4f" depth or
 * ",NaN" off the grid) after the first step ending at or past each multiple of
 * stage_int, and H_final.asc (+ Vx_/Vy_final.asc with voutput) at the end.
 * async_style selects the header of the reference's async writer (xll/yll
 * "%.6f", NODATA "%.0f") rather than its synchronous one ("%.1f", "-9999").
 * Values are formatted exactly as printf("%.4f") does.  With async_style and
 * output_format 1 or 2, each save is also a record of out_dir/output.nc
 * (src/async_output.cpp:20-51, 109-138: time, H and with voutput Vx, Vy as
 * float; NetCDF classic container with 64-bit offsets), and with format 1 the
 * periodic ASC grids are not written.  The GPU keeps stepping while a save is
 * copied out and written by a background thread. */
typedef struct af_output_desc {
  const char* out_dir;   /* dirroot                                            */
  double save_int;       /* saveint; <= 0: no periodic saves                  */
  int voutput;           /* par key voutput                                   */
  int async_style;       /* par key async_output                              */
  double xll, yll;       /* georeference written to the ASC headers           */
  int n_stage;           /* stage points: cell index (-1: off the grid)       */
  const int* stage_idx;
  const char* const* stage_names;  /* NULL entries: "Stage<k>"                */
  double stage_int;      /* par key stageint                                  */
  int output_format;     /* par key output_format: 0 ASC, 1 NetCDF, 2 both;    */
                         /* as in the reference, NetCDF (output.nc, one record */
                         /* per save) only with async_style, and the final     */
                         /* grids are ASC whatever the format                  */
} af_output_desc;

/* Runs to sim_time with the outputs above; *steps (optional) = steps taken. */
int af_sim_run_output(af_sim* s, double sim_time, const af_output_desc* o, int64_t* steps);

/* One ESRI ASCII grid as the reference writes it (row 0 north, values
 * "%.4f " per cell); style 0 = src/io.cpp:314-334's header, 1 = the async
 * writer's (src/async_output.cpp:158-167). */
int af_write_asc(const char* path, const double* values, int ncols, int nrows, double xll,
                 double yll, double cellsize, double nodata, int style);

/* The NetCDF file of the reference's async writer (src/async_output.cpp:20-51,
 * 109-138) from host arrays, for a caller that runs its own loop: dimensions
 * time (unlimited), x, y; time(time) double; H(time, y, x) float (with voutput
 * Vx and Vy too) with the reference's attributes; one record per append,
 * values rounded to float; NetCDF's classic container with 64-bit offsets.
 * The record count in the file is updated after every record.  AF_ERANGE for
 * a grid whose one record of a field exceeds 4 GiB - 4 bytes. */
typedef struct af_netcdf af_netcdf;
int af_netcdf_create(const char* path, int ncols, int nrows, int voutput, double xll, double yll,
                     double cellsize, double nodata, af_netcdf** out);
/* Vx and Vy are read only when the file was created with voutput. */
int af_netcdf_append(af_netcdf* f, double time, const double* H, const double* Vx,
                     const double* Vy);
int af_netcdf_close(af_netcdf* f);

/* ======================================================= 3. batch layer == */

/* No counterpart in the reference, which runs one grid per process: a batch
 * steps many independent grids ("scenarios": own size, parameters, forcing,
 * adaptive dt and stop time) together, one persistent kernel per batch step
 * inside one CUDA graph, each scenario advancing by its own dt exactly as
 * af_sim would step it alone (bit for bit: a scenario's results do not depend
 * on the other members).  Scenarios start at t = 0 (src/main.cpp:197) and
 * stop once t >= t_stop (the loop test of src/main.cpp:227).
 *
 * Device memory: af_batch_create takes one arena of arena_bytes; every
 * scenario's state and tables are placed inside it.  af_batch_add refuses a
 * scenario whose footprint (af_batch_footprint) does not fit in the free
 * arena space with AF_ENOMEM and changes nothing, so a caller admits work by
 * HBM footprint and retries after af_batch_remove frees space.  At most
 * AF_BATCH_MAX_SLOTS scenarios are members at once.
 *
 * One host thread drives a batch.  af_batch_launch enqueues batch steps
 * without waiting; af_batch_sync waits and refreshes the per-slot status that
 * af_batch_slot_status reports.  While a launch is in flight, af_batch_add
 * uploads on a separate copy stream (the scenario joins at the next launch),
 * af_batch_remove defers the release to the next af_batch_sync, and
 * af_batch_get_state works for scenarios that had finished at the last sync. */
#define AF_BATCH_MAX_SLOTS 1024

typedef struct af_batch af_batch;

/* precision: AF_PREC_F32 or AF_PREC_F64.  variant: launch shape of the batch
 * step kernel (0..4: warps per block x resident blocks per SM = 1x16, 1x12,
 * 1x20, 4x4, 2x8), -1 = the default (1x16 in FP32, 1x12 in FP64). */
int af_batch_create(int precision, int device, uint64_t arena_bytes, int variant,
                    af_batch** out);
int af_batch_destroy(af_batch* b);

/* Strip height (rows) used for scenarios of a size class, class =
 * floor(log2(nx*ny)) (0..31).  Applies to scenarios added afterwards; the
 * autotuner sets these.  Results do not depend on the strip height except for
 * the rounding of the volume/area diagnostics. */
int af_batch_size_class(int nx, int ny);
int af_batch_set_rows(af_batch* b, int size_class, int rows);
int af_batch_get_rows(const af_batch* b, int size_class);

/* Arena bytes a scenario would take (fields, tables, reduction and mass-series
 * space) with the batch's precision and current strip heights. */
int af_batch_footprint(const af_batch* b, const af_case_desc* c, const af_forcing_desc* f,
                       double t_stop, uint64_t* bytes);
/* Admits a scenario from HOST arrays (dem, optional h0 as af_sim_create);
 * *slot receives its slot id.  AF_ENOMEM: no room in the arena or no free
 * slot (nothing changed). */
int af_batch_add(af_batch* b, const af_case_desc* c, const af_forcing_desc* f, const double* dem,
                 const double* h0, double t_stop, int* slot);
int af_batch_remove(af_batch* b, int slot);

/* Enqueues batch steps until no member is active, max_steps batch steps have
 * run, (stop_on_done != 0) a scenario has finished, or af_batch_attention is
 * called; does not wait. */
int af_batch_launch(af_batch* b, int64_t max_steps, int stop_on_done);
/* Asks the launch in flight to stop after its current batch step (sets a
 * flag in host memory mapped into the device; safe from any thread). */
int af_batch_attention(af_batch* b);
/* 1 when no launch is in flight or it has finished (af_batch_sync will not
 * wait), 0 while it runs; never waits. */
int af_batch_query(af_batch* b);
/* Waits for the launch; AF_ESTATE if the batch's state is invalid. */
int af_batch_sync(af_batch* b);
/* Steps until every member has finished or max_steps batch steps have run,
 * and waits.  With the load-adaptive strip height on, it launches once per
 * scenario completion so the strips are re-cut for the members that remain. */
int af_batch_run(af_batch* b, int64_t max_steps, int64_t* batch_steps);
/* Load-adaptive strip height: before each launch, the strip height of every
 * active member is the tuned height of its size class, lowered (powers of
 * two, at least 2 rows) until the active members give each warp of the
 * persistent grid about strips_per_warp strips.  0 turns it off (default 4).
 * Results do not depend on it. */
int af_batch_set_balance(af_batch* b, int strips_per_warp);

/* Status of a slot as of the last sync.  *state: 0 running, 1 finished
 * (t >= t_stop), -1 stopped on a bad state (non-finite or non-positive dt). */
int af_batch_slot_status(const af_batch* b, int slot, double* t, double* dt_last, double* hmax,
                         int64_t* steps, int* state);
/* Per-step trace of a batch (no counterpart in the reference: it runs one
 * grid per process).  af_batch_set_trace(b, cap) (re)starts it with room for
 * cap batch steps (0 stops it); af_batch_get_trace copies up to cap records
 * of the steps since then, four int64 each: the step's start and end on the
 * device clock (ns) and the cells and strips it stepped; *n gets how many
 * there are.  Neither may be called while a launch is in flight. */
int af_batch_set_trace(af_batch* b, int64_t cap);
int af_batch_get_trace(af_batch* b, int64_t* rec, int64_t cap, int64_t* n);

/* State of a slot in the reference layout, HOST FP64 arrays (as
 * af_sim_get_state); any pointer may be NULL. */
int af_batch_get_state(af_batch* b, int slot, double* H, double* Qx, double* Qy);
int af_batch_mass_series(af_batch* b, int slot, double* t, double* vol, double* area, int cap,
                         int* n);
int af_batch_info(const af_batch* b, int* members, int64_t* batch_steps, uint64_t* arena_bytes,
                  uint64_t* arena_used, uint64_t* arena_largest_free);
/* The device stream batch launches run on (a cudaStream_t). */
void* af_batch_stream(af_batch* b);

/* The batch's arena planner on its own (host only, no device memory): best-fit
 * placement of 256-byte-aligned blocks in a range of `bytes`, coalescing
 * neighbours on release.  A caller can plan admissions with it. */
typedef struct af_arena af_arena;
int af_arena_create(uint64_t bytes, af_arena** out);
int af_arena_destroy(af_arena* a);
/* AF_ENOMEM when no free block holds `bytes` (nothing changes). */
int af_arena_alloc(af_arena* a, uint64_t bytes, uint64_t* off);
int af_arena_free(af_arena* a, uint64_t off);
int af_arena_stats(const af_arena* a, uint64_t* used, uint64_t* largest_free, int* blocks);

/* ============================================== 4. input files (host) == */

/* A case parsed from a .par file and the files it names, with the
 * reference's parsing rules (src/io.cpp:9-296). */
typedef struct af_scenario af_scenario;

int af_scenario_load(const char* parfile, af_scenario** out);
void af_scenario_free(af_scenario* sc);
/* Views into the parsed case (valid until af_scenario_free).  par[0..2] =
 * sim_time, save_int, mass_int; geo[0..2] = xll, yll, cellsize. */
int af_scenario_get(const af_scenario* sc, af_case_desc* c, af_forcing_desc* f,
                    const double** dem, double* par, double* geo);
/* The case's outputs as the reference's CLI writes them (src/io.cpp:9-47 keys
 * dirroot, saveint, voutput, async_output, output_format, stageint; the stage
 * points of stagefile read as src/io.cpp:50-85 does), for af_sim_run_output;
 * the strings and arrays stay valid until af_scenario_free. */
int af_scenario_output(const af_scenario* sc, af_output_desc* o);

#ifdef __cplusplus
}
#endif
#endif /* ADAPTFLOOD_H */
