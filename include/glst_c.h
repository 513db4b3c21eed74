/*
 * glst_c.h -- C-ABI of the B200-native GLST electrostatics engine.
 *
 * One opaque handle replaces one `glst_force<CT>` object of the reference
 * library (include/glst_force.hcu:24-125).  Every entry point takes plain
 * pointers and sizes; CUDA streams are passed as `void*` (a cudaStream_t, or
 * NULL for the legacy default stream).  No C++ or torch types cross this
 * boundary and no exception escapes it: every call returns a glst_status and
 * glst_last_error() gives the message of the last failure on this thread.
 *
 * Physics (same as the reference): open-boundary Coulomb energy and forces of
 * point charges, in units of e^2/A (no Coulomb constant).  en[i] counts every
 * pair from both sides, so the total energy is 0.5 * sum(en) (glst_energy).
 *
 * Differences from the reference's behaviour, all deliberate:
 *   - outputs are overwritten by every compute call (the reference adds into
 *     fx_/fy_/fz_/en_ and its caller zeroes them, test/full_example.cu:201-209);
 *   - the compute path is fully stream ordered and never blocks the host
 *     (the reference copies cell counts to the host every step,
 *     src/glst_force.cu:474-482), so it can be captured in a CUDA graph;
 *   - CUDA errors are always checked and returned (the reference ignores them
 *     in release builds, include/cuda_utils.hcu:38-42).
 */
#ifndef GLST_C_H
#define GLST_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum glst_status {
  GLST_OK = 0,
  GLST_ERR_INVALID_ARG = 1,   /* bad pointer, size or parameter */
  GLST_ERR_CUDA = 2,          /* a CUDA runtime call failed */
  GLST_ERR_NO_DEVICE = 3,     /* no CUDA device */
  GLST_ERR_TDESIGN = 4,       /* spherical t-design store missing / degree absent */
  GLST_ERR_NO_CONVERGENCE = 5,/* GL rule / t-design / erfc inverse not found */
  GLST_ERR_OUT_OF_MEMORY = 6, /* device allocation failed */
  GLST_ERR_SIZE = 7,          /* a size limit of this build was exceeded */
  GLST_ERR_STATE = 8          /* call out of order (e.g. get_ef before compute) */
} glst_status;

/* Calculation type of the reference object this handle stands in for.  It
 * selects how the cell grid and the cell of each atom are computed (in float
 * or double, src/glst_force.cu:223-241, :356-386) and the type the cubature
 * nodes are rounded to (src/cubature.cu:138-141), so that the cell assignment
 * is bit-identical to glst_force<float> or glst_force<double>.  The arithmetic
 * of the sum itself is this engine's mixed precision in both cases. */
typedef enum glst_ct { GLST_CT_DOUBLE = 0, GLST_CT_FLOAT = 1 } glst_ct;

typedef struct glst_handle glst_handle;

/* Plan summary (what the reference prints from init, src/glst_force.cu:245-293). */
typedef struct glst_info {
  uint32_t natom;
  uint32_t ncell[3];
  uint32_t ncell_total;
  double cell_dim;          /* cell edge as the CT value, widened to double */
  uint32_t ngroup;          /* alpha groups */
  uint32_t num_nodes;       /* K, total cubature nodes */
  uint32_t has_far_field;   /* 0 when some dimension has <= 2 cells */
  uint32_t group_nodes[16]; /* nodes per group (first 16 groups) */
  uint32_t group_gl_degree[16];
  uint32_t group_t_degree[16];
  double group_alpha[16];
  double group_zcut[16];
  double group_rmax[16];
  uint32_t group_r_in[16];
  uint32_t group_r_out[16];
  uint64_t device_bytes;    /* device memory held by the handle */
  uint32_t kernels_per_compute; /* kernel launches of one glst_compute */
  uint32_t node_stages;     /* far-field node stages of one compute: the
                               structure factors and shell sums of a stage's
                               nodes are held at a time (large systems hold a
                               fraction of the ncell x K operand) */
  uint32_t shell_sums_form; /* 0: prefix tables in shared memory, one or more
                               nodes per CTA; 1: the grid's per-node table
                               does not fit in shared memory, tables in global
                               memory (any grid size) */
  uint32_t gather_variant;  /* share of the gather's sines/cosines on the FMA
                               pipe: 0 = 2 in 14 node pairs (default), 1 =
                               none, 2 = 1 in 14, 3 = 3 in 14 (glst_autotune) */
  uint32_t sf_max_npt;      /* radial nodes per thread, at most, in the
                               structure-factor units (12 by default;
                               glst_autotune) */
} glst_info;

/* Where spherical t-designs are read from.  Either the project's binary store
 * (tdesigns.bin) or a directory in the reference's text layout (the
 * reference reads "SS31-Mar-2016/" in the working directory,
 * src/cubature.cu:423-459, :490).  Default: the environment variable
 * GLST_TDESIGN_PATH, else "SS31-Mar-2016/" if it exists in the working
 * directory, else the store shipped next to the library.  Process-wide. */
glst_status glst_set_tdesign_path(const char *path);

/* glst_force(natom, tol, Lx, Ly, Lz, rcut)   src/glst_force.cu:72-78
 * Plans cells, alpha groups and the cubature on the host (FP64) and
 * allocates all device buffers on the current device. */
glst_status glst_create(glst_handle **out, uint32_t natom, double tol,
                        double box_x, double box_y, double box_z, double rcut,
                        glst_ct ct);

/* glst_force(natom, tol, Lx, Ly, Lz, ncx, ncy, ncz)   src/glst_force.cu:80-95
 * rcut = min(L/n) over the three axes. */
glst_status glst_create_ncell(glst_handle **out, uint32_t natom, double tol,
                              double box_x, double box_y, double box_z,
                              uint32_t ncell_x, uint32_t ncell_y,
                              uint32_t ncell_z, glst_ct ct);

/* One device's share of a system split over several GPUs, the reference's
 * multi-GPU scheme (src/glst_force.cu:276-293 node split, :1584-1602 reduce):
 * shard s of n computes the structure factors, shell sums and long-range
 * gather of a contiguous range of about K/n cubature nodes, and shard 0 also
 * the near field.  The per-atom outputs of the n shards add up to the full
 * result; sum them across devices (e.g. ncclAllReduce of fx, fy, fz, en) --
 * the engine does no communication.  Otherwise as glst_create. */
glst_status glst_create_shard(glst_handle **out, uint32_t natom, double tol,
                              double box_x, double box_y, double box_z,
                              double rcut, glst_ct ct, uint32_t shard,
                              uint32_t nshards);

/* The reference's reduction of the shards' partial results to the first GPU
 * (comm_ef, src/glst_force.cu:1584-1602: ncclReduce of fx, fy, fz, en to
 * device 0, src/device_comm.cu:176-201).  shards[s] is shard s of n of one
 * system (glst_create_shard), each after its glst_compute on streams[s]
 * (its own device).  Shard 0's device reads the other shards' outputs
 * directly over NVLink (peer access, enabled here when the devices differ)
 * and sums them in shard order into shard 0's outputs, input and cell order,
 * and its total energy; glst_get_ef / glst_energy on shard 0 then return
 * the whole system's result.  Stream ordered on streams[0], which first waits
 * for every shard's stream.  At most 16 shards. */
glst_status glst_reduce_shards(glst_handle *const *shards, uint32_t n,
                               void *const *streams);

/* glst_force::init(natom, tol, Lx, Ly, Lz, rcut)   src/glst_force.cu:179-327 */
glst_status glst_init(glst_handle *h, uint32_t natom, double tol, double box_x,
                      double box_y, double box_z, double rcut);

/* ~glst_force()   src/glst_force.cu:97-100, :1768-1796 */
glst_status glst_destroy(glst_handle *h);

/* glst_force::calc_ener_force(d_rx, d_ry, d_rz, d_qc)   src/glst_force.cu:1604-1614
 * Device pointers to natom FP64 values each (positions in A, charges in e),
 * caller owned, read during the call only.  Stream ordered; returns without
 * waiting for the GPU. */
glst_status glst_compute(glst_handle *h, const double *d_rx, const double *d_ry,
                         const double *d_rz, const double *d_qc, void *stream);

/* The six phases of calc_ener_force, for callers of the reference's phase
 * methods (include/glst_force.hcu:52-58).  Run in this order they produce
 * exactly what glst_compute produces.  When the far field runs in several
 * node stages (glst_info.node_stages > 1; the structure factors and shell
 * sums of one stage are held at a time), glst_calc_sf runs the whole far
 * field stage by stage and glst_sum_rmt_sf / glst_calc_lr_ef return at once. */
glst_status glst_assign_atoms(glst_handle *h, const double *d_rx,
                              const double *d_ry, const double *d_rz,
                              const double *d_qc, void *stream); /* :431-534 */
glst_status glst_calc_sf(glst_handle *h, void *stream);      /* :666-700 */
glst_status glst_sum_rmt_sf(glst_handle *h, void *stream);   /* :915-981 */
glst_status glst_calc_lr_ef(glst_handle *h, void *stream);   /* :1137-1168 */
glst_status glst_calc_sr_ef(glst_handle *h, void *stream);   /* :1546-1582 */
glst_status glst_comm_ef(glst_handle *h, void *stream);      /* :1584-1602 */

/* glst_force::get_ef(fx, fy, fz, en)   src/glst_force.cu:142-176
 * Copies forces and per-atom energies in INPUT order into the four arrays
 * (natom doubles each).  `on_device` = 0: host pointers, the call waits for
 * the stream; 1: device pointers, stream ordered.  Any pointer may be NULL. */
glst_status glst_get_ef(glst_handle *h, double *fx, double *fy, double *fz,
                        double *en, int on_device, void *stream);

/* Device pointers to the CELL-ordered outputs, as the reference's
 * fx()/fy()/fz()/en() accessors return them (include/glst_force.hcu:36-43). */
glst_status glst_cell_outputs(glst_handle *h, double **fx, double **fy,
                              double **fz, double **en);

/* Total energy 0.5 * sum_i en_i, reduced on the device in a fixed order
 * (waits for the stream).  The reference leaves this sum to its caller. */
glst_status glst_energy(glst_handle *h, double *e_total, void *stream);

/* End to end from HOST memory: copies positions and charges to the device,
 * computes, and copies forces/energies (input order) back; waits for the
 * stream.  Equivalent to H2D + glst_compute + glst_get_ef(on_device=0). */
glst_status glst_compute_host(glst_handle *h, const double *rx,
                              const double *ry, const double *rz,
                              const double *qc, double *fx, double *fy,
                              double *fz, double *en, void *stream);

/* Cell assignment of the last compute, copied to host arrays (waits):
 * sorted_idx[natom] = input index of the atom at each cell-ordered slot
 * (the reference's sorted_idx_), cell_count/cell_point[ncell] (its
 * cell_atom_count_/cell_atom_point_).  Any pointer may be NULL. */
glst_status glst_get_assignment(glst_handle *h, uint32_t *sorted_idx,
                                uint32_t *cell_count, uint32_t *cell_point);

glst_status glst_get_info(const glst_handle *h, glst_info *info);

/* Cubature node set in the reference's order (group, radial, direction;
 * src/cubature.cu:120-145), FP64 before any rounding to CT.  Arrays of
 * info.num_nodes; any pointer may be NULL. */
glst_status glst_get_nodes(const glst_handle *h, double *kx, double *ky,
                           double *kz, double *w, uint32_t *group);

/* Host-only planning, no device needed: the same cell grid, alpha groups and
 * cubature glst_create would build (src/glst_force.cu:179-327).  Fills *info
 * (device_bytes = 0) and, when non-NULL, the node arrays (info->num_nodes
 * entries each; call once with NULL arrays to learn the count). */
glst_status glst_plan(uint32_t natom, double tol, double box_x, double box_y,
                      double box_z, double rcut, glst_ct ct, glst_info *info,
                      double *kx, double *ky, double *kz, double *w,
                      uint32_t *group);

/* Autotuner: times, on these inputs (device FP64 arrays, as glst_compute),
 * the shell-sum kernel for 1..32 nodes per CTA, the long-range gather for
 * 2..32 waves of chunk CTAs and for each of its compiled FMA-pipe sine/cosine
 * shares, and the structure factors for 12 / 8 / 6 radial nodes per thread;
 * keeps the fastest for this handle, and remembers them for every later
 * handle of the same shape (cells, nodes, atom-count bucket) in this process.
 * Returns the first two choices (glst_get_info reports the others).  Waits for
 * the stream; outputs must be recomputed afterwards.  Handles whose far field
 * runs in one node stage only.  No reference counterpart. */
glst_status glst_autotune(glst_handle *h, const double *d_rx,
                          const double *d_ry, const double *d_rz,
                          const double *d_qc, void *stream, uint32_t *sat_nb,
                          uint32_t *lr_waves);

/* Direct all-pairs Coulomb energies and forces in FP64, open boundary: the
 * reference's physics check (utils/coulomb.cu:14-172, compute_coulomb_cuda),
 * on the current device.  Device arrays of natom doubles, input order; en
 * counts each pair from both sides like the GLST outputs.  Stream ordered;
 * O(natom^2) work, meant for checking systems up to ~1e5 atoms. */
glst_status glst_direct_coulomb(uint32_t natom, const double *d_rx,
                                const double *d_ry, const double *d_rz,
                                const double *d_qc, double *d_fx, double *d_fy,
                                double *d_fz, double *d_en, void *stream);

/* Measured pipe peaks of the current device, the denominators of the
 * roofline of the phase kernels (which are bound by the SFU sin/cos and FP32
 * pipes, not by tensor cores or HBM): `sfu_per_s` = MUFU sin+cos results per
 * second, `fma_per_s` = FP32 fused multiply-adds per second, each from a
 * dependent-chain loop over every SM.  Waits for the device. */
glst_status glst_measure_pipe_peaks(double *sfu_per_s, double *fma_per_s);

/* Device-side error flags raised by the last compute (none are raised by
 * this build's kernels; GLST_ERR_STATE if any is set).  Waits for the stream. */
glst_status glst_check(glst_handle *h, void *stream);

/* Atoms per cell the shared-memory cell sort holds.  Larger cells are
 * ordered by a slower pass over all atoms; the assignment stays identical to
 * the reference's (stable order by input index) at any cell size. */
uint32_t glst_max_atoms_per_cell(void);

/* Structure factors and shell sums of the positions last assigned (by
 * glst_compute or glst_assign_atoms), recomputed stage by stage and returned
 * in the reference's layout and definitions: host arrays of ncell x K
 * doubles, row = cell, nodes in the reference's order (glst_get_nodes);
 * sf = sum_j q_j e^{-i k.r_j} (the reference's sf_re_/sf_im_ after calc_sf,
 * src/glst_force.cu:601-664) and rmt = w_k times the shell sum (its
 * rmt_sum_re_/rmt_sum_im_ after sum_rmt_sf, :774-913).  This engine stores
 * them cell-relative and pre-twiddled in FP32; the conversion is FP64 on the
 * host.  For checking the two far-field phases separately; whole-system
 * handles only (not shards).  Any pointer may be NULL; waits for the stream.
 * No counterpart in the reference's public interface (the arrays are private
 * members there). */
glst_status glst_get_far_field(glst_handle *h, double *sf_re, double *sf_im,
                               double *rmt_re, double *rmt_im, void *stream);

/* ---------------------------------------------------------------------------
 * Batches: many independent systems solved together.  No counterpart in the
 * reference (one system per glst_force object).  Each system keeps its own
 * plan and buffers; one compute runs all of them as one CUDA graph whose
 * branches (nstreams concurrent streams, systems assigned largest-first) fill
 * the GPU with systems of uneven size.  Inputs/outputs are concatenated in
 * system order: system i owns entries [off_i, off_i + natom_i), off_i the
 * prefix sum of natom.
 * ------------------------------------------------------------------------- */
typedef struct glst_batch glst_batch;

glst_status glst_batch_create(glst_batch **out, uint32_t nsys,
                              const uint32_t *natom, const double *tol,
                              const double *box /* 3 per system */,
                              const double *rcut, glst_ct ct,
                              uint32_t nstreams);
glst_status glst_batch_destroy(glst_batch *b);

/* Solve every system.  `plain` selects the schedule:
 *   0: one captured CUDA graph (captured on the first call and again whenever
 *      the pointers or the mode change) of every system's own launch
 *      sequence, spread over `nstreams` parallel branches (systems assigned
 *      largest first to the least loaded branch, those that fill the GPU
 *      alone on one branch) -- the fastest schedule measured;
 *   1: the systems one after another on one stream, each its own launch
 *      sequence (the one-system-per-launch baseline);
 *   2: one captured graph in which every system that fits the work-list
 *      kernels (whole system, one node stage, shell sums in shared memory,
 *      default launch variants) is solved by one launch per phase --
 *      assignment, structure factors, shell sums, gather, near field,
 *      combine -- over a work list of (system, unit / cell / node block /
 *      atom block x chunk) items, each item running exactly the code the
 *      system's own launch would (in groups on parallel branches); the other
 *      systems run their own launch sequences beside them.
 * Every mode gives every system bit for bit the result it gets alone.
 * Outputs in input order per system.  Stream ordered. */
glst_status glst_batch_compute(glst_batch *b, const double *d_rx,
                               const double *d_ry, const double *d_rz,
                               const double *d_qc, double *d_fx, double *d_fy,
                               double *d_fz, double *d_en, int plain,
                               void *stream);

/* Total energy of every system (nsys doubles, host), waits for the stream. */
glst_status glst_batch_energies(glst_batch *b, double *e, void *stream);

/* Handle of system i (owned by the batch; do not destroy): its plan
 * (glst_get_info) and cell-ordered outputs.  A batched solve writes the
 * input-order outputs and the total energy straight into the batch's arrays
 * (glst_batch_compute's outputs, glst_batch_energies), not into the handle. */
glst_status glst_batch_system(glst_batch *b, uint32_t i, glst_handle **h);

/* ---------------------------------------------------------------------------
 * Request server: energy+force requests of independent systems served with
 * continuous batching.  No counterpart in the reference.  A worker thread
 * admits queued requests as soon as a stream slot is free and the systems'
 * device memory fits the budget (idle resident systems are evicted least
 * recently used first), runs each on its own stream (H2D from pinned
 * staging, solve, D2H), and completes them as their events fire.  A request
 * naming a resident system (same key, natom, tol, box, rcut) reuses its plan
 * and buffers: only positions and charges move.
 * ------------------------------------------------------------------------- */
typedef struct glst_server glst_server;

typedef struct glst_server_stats {
  uint64_t submitted, completed, evictions, systems_created;
  uint64_t resident_bytes, peak_resident_bytes;
  uint32_t resident_systems, in_flight;
} glst_server_stats;

/* budget_bytes: device memory the resident systems may hold; nslots:
 * requests in flight at once (1 = one request at a time). */
glst_status glst_server_create(glst_server **out, uint64_t budget_bytes,
                               uint32_t nslots);
glst_status glst_server_destroy(glst_server *s);

/* Queue a request; inputs are copied before the call returns.  `key` names
 * the system (0 = a new, unnamed system, freed after the request).  Returns a
 * ticket.  Host arrays of natom doubles. */
glst_status glst_server_submit(glst_server *s, uint64_t key, uint32_t natom,
                               double tol, double box_x, double box_y,
                               double box_z, double rcut, const double *rx,
                               const double *ry, const double *rz,
                               const double *qc, uint64_t *ticket);

/* Wait for a request (timeout_ms < 0: no limit; returns GLST_ERR_STATE on
 * timeout), copy its outputs (input order, host, any may be NULL), total
 * energy and latency (submit to completion, microseconds), and forget it. */
glst_status glst_server_wait(glst_server *s, uint64_t ticket, double *fx,
                             double *fy, double *fz, double *en,
                             double *energy, double *latency_us,
                             double timeout_ms);

glst_status glst_server_get_stats(glst_server *s, glst_server_stats *st);

/* Near-field energies and forces WITHOUT ALLOCATING DEVICE MEMORY.  No
 * counterpart in the reference.  For callers that cannot call cudaMalloc when
 * they need forces: code that runs while a stream is being captured into a
 * CUDA graph (allocation is not allowed during capture), and engines or
 * plugins whose host owns the whole device through its own memory pool.
 * Computes the reference's near field -- bare Coulomb over the own cell and
 * the 26 neighbour cells of the grid built from (box, rcut, ct), open
 * boundary -- which is the complete GLST result when some axis has at most 2
 * cells (the reference then has no far field, src/glst_force.cu:667-670).
 * Inputs d_rx..d_qc and outputs d_fx..d_en (input order) are natom device
 * doubles owned by the caller.  Working memory is one file-scope __device__
 * array of GLST_NOALLOC_SCRATCH_BYTES, present on every GPU that loads the
 * library until the process exits; sizes above GLST_NOALLOC_MAX_ATOMS atoms or
 * GLST_NOALLOC_MAX_CELLS cells return GLST_ERR_SIZE.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress, device
 * current); make that first call before any stream capture.  All calls share
 * the array: calls that overlap on the GPU (different streams or devices'
 * threads racing on one device) corrupt each other; serialise them.  Stream
 * ordered, does not wait for the GPU.  The cell assignment is the
 * reference's at any cell size. */
#define GLST_NOALLOC_MAX_ATOMS 32768u
#define GLST_NOALLOC_MAX_CELLS 32768u
#define GLST_NOALLOC_SCRATCH_BYTES 6561792ull
glst_status glst_near_field_noalloc(uint32_t natom, const double *d_rx,
                                    const double *d_ry, const double *d_rz,
                                    const double *d_qc, double box_x,
                                    double box_y, double box_z, double rcut,
                                    glst_ct ct, double *d_fx, double *d_fy,
                                    double *d_fz, double *d_en, void *stream);

const char *glst_last_error(void);
const char *glst_status_string(glst_status s);
const char *glst_version(void);

#ifdef __cplusplus
}
#endif
#endif /* GLST_C_H */
