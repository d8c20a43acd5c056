/*
 * lbm_b200.h — C ABI of the B200 D3Q19 lattice-Boltzmann time step.
 *
 * This is the drop-in boundary for the hot path of NFLOW-RED-Poplar (the
 * E8ight LBM3D solver ported to Poplar).  Every entry point below names the
 * reference interface it replaces (file:line inside the reference project).
 * Plain C types only: pointers, sizes and the reference's own Inputval
 * struct, so the header can be bound from C, C++ (lbm_b200_compat.hpp adds
 * the reference's C++ names), ctypes or any other FFI.
 *
 * Conventions kept from the reference
 *   - axis order [y][z][x], y slowest: node id = x + z*nx + y*nx*nz
 *     (main.cpp:1, lbm_codelets.cpp:52);
 *   - D3Q19 velocity ordering, opposite table and weights of main.cpp:87-146;
 *   - the population array arF at the boundary is AoS with the direction
 *     fastest: arF[dir + node*19].  Two views are offered:
 *       unpadded  [ny][nz][nx][19]          (main.cpp:216, the tensor main.cpp
 *                                            writes with "H2D-arF" and reads
 *                                            back with "D2H-arF"),
 *       padded    [ny+2][nz+2][nx+2][19]    (README "Output sliced Tensor",
 *                                            one ghost layer per side; the
 *                                            ghost layer is written as 0).
 *   Internally populations live on the GPU in a private SoA layout; the
 *   AoS<->SoA transform happens only at import/export.
 *
 * Error handling: every call returns an int status (LBM_OK == 0, negative
 * on failure) and lbm_last_error() returns a per-thread message.  Nothing
 * calls exit(); the reference exits on a singular MRT matrix
 * (inverseMRT.cpp:86-90) and on fopen failures (kernel.cu:711, 979).
 *
 * Threading: a domain handle may be used by one host thread at a time.
 * All device work of a handle is ordered on the handle's CUDA stream
 * (lbm_set_stream); calls that return host data synchronise that stream.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>
#include <stdint.h>
#ifndef __cplusplus
#include <stdbool.h>
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Parameters of common.h:7-39 (same names and values).                */
/* ------------------------------------------------------------------ */
#ifndef DIMENSION
#define DIMENSION 3
#endif
#ifndef DIRECTION_SIZE
#define DIRECTION_SIZE 19
#endif
#ifndef XDIM
#define XDIM 0
#define ZDIM 1
#define YDIM 2
#endif
#ifndef XDECOMP
#define XDECOMP 3
#define YDECOMP 3
#define ZDECOMP 3
#endif
#ifndef CAVITY
#define CAVITY 1
#define POISEUILLE 0
#endif
/* Extension: straight channel, parabolic velocity inlet at x=0, constant
 * pressure outlet at x=nx-1, bounce-back walls on the four side faces. */
#ifndef CHANNEL
#define CHANNEL 2
#endif
#ifndef NODE_FLUID
#define NODE_FLUID (1 << 1)
#define NODE_FIXEDWALL (1 << 2)
#define NODE_MOVINGWALL (1 << 3)
#define NODE_INLET (1 << 4)
#define NODE_OUTLET (1 << 5)
#define NODE_STRUCT (1 << 6)
#endif
#ifndef TILE_NUM
#define TILE_NUM 1471
#endif

/* ------------------------------------------------------------------ */
/* struct.h:78-100 Inputval, field for field (same order and types).    */
/* `length` is a float in the reference; this library never reads it    */
/* and sizes every array from nx*ny*nz instead.                          */
/* ------------------------------------------------------------------ */
#ifndef LBM_INPUTVAL_DEFINED
#define LBM_INPUTVAL_DEFINED
typedef struct Inputval {
  int h;
  int nx, ny, nz;
  int ngrid;
  int maxitr;
  int nwrite, irestart, irst;
  int icycle;
  float m_dSmagorinsky;
  float Re, length, nu;
  float m_dRefViscosity;
  float m_dRefDen;
  float m_dTau;
  float m_dRefVelx, m_dRefVely, m_dRefVelz;
  float dWeps, dWepsj, dWXX;
  bool bEnableMRT;
  bool bEnableLES;
  int savetype;
  int casetype;
} Inputval;
#endif

/* ------------------------------------------------------------------ */
/* Status codes                                                         */
/* ------------------------------------------------------------------ */
enum {
  LBM_OK = 0,
  LBM_ERR_INVALID = -1,   /* bad argument, size or configuration          */
  LBM_ERR_CUDA = -2,      /* a CUDA runtime/driver call failed            */
  LBM_ERR_OOM = -3,       /* device allocation failed                      */
  LBM_ERR_SINGULAR = -4,  /* MRT matrix not invertible                     */
  LBM_ERR_STATE = -5,     /* call not valid in the handle's current state  */
  LBM_ERR_TIMEOUT = -6,   /* a bounded device wait gave up                 */
  LBM_ERR_BUDGET = -7,    /* request exceeds the HBM budget                */
  LBM_ERR_NOT_FINITE = -8,/* input data holds NaN/Inf                      */
  LBM_ERR_NO_DEVICE = -9, /* no CUDA device / extension not usable         */
  LBM_ERR_IO = -10        /* an output file could not be written          */
};

/* Population storage of a domain (all arithmetic is done in FP32 except
 * LBM_STORE_F64, which is the double-precision build used as the oracle
 * on the GPU).  The *_SHIFT forms store f_i - w_i (times a per-domain
 * power-of-two scale) so that the 16-bit format holds the deviation from
 * the rest state, not the value itself. */
enum {
  LBM_STORE_F32 = 0,
  LBM_STORE_F16_SHIFT = 1,
  LBM_STORE_BF16_SHIFT = 2,
  LBM_STORE_F64 = 3
};

/* Initial condition.  LBM_INIT_REFERENCE reproduces the Initialize
 * codelet (lbm_codelets.cpp:140-241) / keInitialize (kernel.cu:282-315):
 * rho = RefDen, u = 0 except the lid (cavity) nodes.  The two seeded forms
 * add a deterministic counter-based perturbation (splitmix64 of the node id)
 * so that the CPU oracle and the GPU produce identical initial bits. */
enum {
  LBM_INIT_REFERENCE = 0,
  LBM_INIT_DENSITY_NOISE = 1,   /* rho = RefDen + amp*U(-1,1)                */
  LBM_INIT_CHANNEL = 2          /* u = inlet profile + amp*u_max*U(-1,1) per */
                                /* component on non-wall nodes, rho = RefDen */
};

/* Streaming schedule of the fused kernel. */
enum {
  LBM_STREAM_AB = 0,   /* pull, two population lattices (A/B)             */
  LBM_STREAM_AA = 1    /* in-place AA pattern, one lattice (half memory);
                          CAVITY and CHANNEL cases, alone or as batch
                          members (not with a solid mask)                   */
};

/* Kernel variant of the fused step (FP32-arithmetic storage formats). */
enum {
  LBM_KERNEL_AUTO = 0,    /* the fastest variant for the format             */
  LBM_KERNEL_SCALAR = 1,  /* one node per thread                            */
  LBM_KERNEL_PACKED = 2,  /* two nodes per thread, packed FP32 arithmetic   */
  LBM_KERNEL_TMA = 3,     /* TMA-staged tiles, persistent producer/consumer */
  LBM_KERNEL_PAIRED = 4,  /* 16-bit pull form: rows stored as 32-bit words of
                             the node pairs (x, x + px/2), two nodes per thread
                             with packed FP32 arithmetic; the default (AUTO)
                             of FP16/BF16 shifted storage with LBM_STREAM_AB  */
  LBM_KERNEL_QUAD = 5     /* 16-bit AA form: rows stored as 8-byte words of
                             the nodes (w, w + nx/2, w + nx/4, w + 3nx/4), four
                             nodes per thread, every access an aligned 8-byte
                             word in both AA step kinds; the default (AUTO) of
                             FP16/BF16 shifted storage with LBM_STREAM_AA when
                             nx is a multiple of 8 and at least 16            */
};

typedef struct lbm_options {
  int storage;          /* LBM_STORE_*                                     */
  int init_kind;        /* LBM_INIT_*                                      */
  uint64_t seed;        /* perturbation seed                               */
  float noise_amp;      /* perturbation amplitude (see LBM_INIT_*)         */
  float store_scale;    /* *_SHIFT storage scale; 0 = automatic            */
  int stream_mode;      /* LBM_STREAM_*                                    */
  int device;           /* CUDA device ordinal                             */
  int kernel;           /* LBM_KERNEL_*                                    */
  int rounding;         /* LBM_ROUND_*: rounding of the 16-bit stores      */
  int wait_test;        /* test of the bounded waits, LBM_KERNEL_TMA only:
                           k > 0 makes the TMA producer withhold the copies
                           of tile k-1 and every wait give up after ~1 ms,
                           so that the step reports LBM_ERR_TIMEOUT; 0 off */
  int reserved[5];
} lbm_options;

/* Rounding of the shifted 16-bit stores.  NEAREST: round to nearest even.
 * STOCHASTIC: each stored deviation rounds up or down with probability
 * given by its position between the two neighbouring 16-bit values
 * (unbiased: the expected stored value is the exact one), with random bits
 * from a hash of (node pair, step, seed), so runs are reproducible.  In a
 * steady flow round-to-nearest rounds the same value the same way every
 * step, a bias that accumulates; stochastic rounding turns it into noise.
 * STOCHASTIC needs FP16/BF16 shifted storage, with LBM_STREAM_AB and kernel
 * AUTO, PAIRED or SCALAR, or with LBM_STREAM_AA on quad rows (kernel AUTO or
 * QUAD) (single domains; batch members round to nearest).  The initial
 * state, imports and the first AA step after the initial state round to
 * nearest. */
enum { LBM_ROUND_NEAREST = 0, LBM_ROUND_STOCHASTIC = 1 };

/* Fill *opt with the defaults: FP32, reference init, A/B streaming. */
void lbm_default_options(lbm_options* opt);

/* Message of the last failed call made on this host thread. */
const char* lbm_last_error(void);

/* Library version string. */
const char* lbm_version(void);

/* ------------------------------------------------------------------ */
/* Host numerics (no GPU needed).                                       */
/* ------------------------------------------------------------------ */

/* Replaces `int decomposition(Inputval*, int Slice[][3][2])`
 * (decomposition.cpp:98-161): cut the domain into XDECOMP*YDECOMP*ZDECOMP
 * chunks; Slice[t][dim][0/1] = start/end with dim 0=x, 1=y, 2=z.
 * Returns the tile count (>= 0) or a negative status.  On the GPU these
 * chunks become the CTA work-list of the fused kernel. */
int lbm_decomposition(const Inputval* pinput, int Slice[][DIMENSION][2]);

/* Replaces `int set_move_decomp(int NTILE, const int Slice[][3][2],
 * int Move[][19])` (decomposition.cpp:17-62): per tile, the offset of each
 * neighbour inside the tile's ghost-padded slice.  Returns 0. */
int lbm_set_move_decomp(int NTILE, const int Slice[][DIMENSION][2],
                        int Move[][DIRECTION_SIZE]);

/* Replaces `int slice_chunk(unsigned tile, const int Slice[][3][2], int *xs,
 * int *xe, int *ys, int *ye, int *zs, int *ze, int *chunk_nx, int *chunk_ny,
 * int *chunk_nz, int *chunk_len)` (decomposition.cpp:66-94).  Returns 1 when
 * the tile is empty (skip it), 0 otherwise. */
int lbm_slice_chunk(unsigned tile, const int Slice[][DIMENSION][2], int* xs,
                    int* xe, int* ys, int* ye, int* zs, int* ze, int* chunk_nx,
                    int* chunk_ny, int* chunk_nz, int* chunk_len);

/* Replaces `void inverseMRT(vector<vector<float>>&, vector<vector<float>>&)`
 * (inverseMRT.cpp:8-92): Gauss-Jordan inverse in FP32 with the same pivot
 * row rotation.  mat/inv are row-major 19x19.  Returns LBM_ERR_SINGULAR
 * instead of exit(0). */
int lbm_inverse_mrt(const float* mat, float* inv);

/* The D3Q19 tables of main.cpp:87-146 and the moment matrix of
 * main.cpp:149-171: direction[3*19] (rows X, Z, Y as in the reference's
 * flat Direction tensor), opp[19], w[19], M[19*19] row-major.  Any pointer
 * may be NULL. */
void lbm_d3q19_tables(float* direction, int* opp, float* w, float* M);

/* ------------------------------------------------------------------ */
/* Single domain on one GPU.                                            */
/* ------------------------------------------------------------------ */
typedef struct lbm_domain lbm_domain;

/* Allocate a domain for the case in *pinput (nx, ny, nz, casetype, tau,
 * Smagorinsky constant, reference density/velocity, MRT/LES switches) and
 * build its constant tables.  opt may be NULL (defaults). */
int lbm_create(const Inputval* pinput, const lbm_options* opt,
               lbm_domain** out);

/* Free all device memory of the handle. */
int lbm_destroy(lbm_domain* d);

/* Use this CUDA stream (a cudaStream_t passed as void*; NULL is the CUDA
 * default stream, as everywhere in CUDA) for all later work of the handle.
 * A new handle uses its own non-blocking stream. */
int lbm_set_stream(lbm_domain* d, void* cuda_stream);

/* The handle's current CUDA stream (as void*). */
void* lbm_get_stream(lbm_domain* d);

/* Replaces the `initialize` program (initialize.cpp:23-98, the Initialize
 * compute set) and the icycle==0 branch of kernel.cu:156-164: node types,
 * direction masks and the equilibrium populations, on the device. */
int lbm_initialize(lbm_domain* d);

/* Replaces the `runSimulation` program (runSimulation.cpp:22-168) repeated
 * nsteps times (main.cpp:290-291 Repeat(maxitr, ...)), and the else-branch
 * of kernel.cu:166-200.  One fused kernel per step: streaming + boundary
 * conditions + macroscopic + LES + SRT/MRT collision.  Asynchronous. */
int lbm_run_simulation(lbm_domain* d, int nsteps);

/* Steps completed since the last initialize/import. */
int lbm_steps_done(const lbm_domain* d, long long* steps);

/* engine.writeTensor("H2D-arF", ...) (main.cpp:303) followed by a restart
 * from that state: host AoS populations -> device.  padded != 0 selects the
 * [ny+2][nz+2][nx+2][19] view (ghost layer ignored).  The macroscopic
 * fields are recomputed from the imported populations. */
int lbm_import_arF(lbm_domain* d, const float* arF, int padded);

/* engine.readTensor("D2H-arF", ...) (main.cpp:317): the post-streaming,
 * post-boundary populations after the last step, device -> host AoS. */
int lbm_export_arF(lbm_domain* d, float* arF, int padded);

/* CurrDen / CurrVelx / CurrVely / CurrVelz after the last step (the
 * Macroscopic codelet, lbm_codelets.cpp:248-318), [ny][nz][nx] each.
 * Any pointer may be NULL. */
int lbm_get_macroscopic(lbm_domain* d, float* den, float* velx, float* vely,
                        float* velz);

/* NodeType (common.h:32-37 bits) and DirectionState (19-bit inside mask,
 * lbm_codelets.cpp:163-178) per node, [ny][nz][nx]. Either may be NULL. */
int lbm_get_node_info(lbm_domain* d, int* node_type, int* direction_state);

/* Diagnostics of the state after the last step, reduced on the device in
 * FP64 with a fixed order (bit-reproducible):
 *   out[0] = mass        sum rho
 *   out[1..3] = momentum sum rho*u
 *   out[4] = L1 residual sum |rho - rho_prev| over the last step
 *            (kernel.cu:232-248 prints the same quantity)
 *   out[5] = kinetic energy 0.5*sum rho*|u|^2
 *   out[6] = max |u|
 *   out[7] = number of non-finite populations (0 when healthy)
 * Synchronises the handle's stream. */
int lbm_diagnostics(lbm_domain* d, double out[8]);

/* Solid voxels (general solid masks: keBoundaryStruct, kernel.cu:659-697,
 * on any geometry).  mask[ny][nz][nx], nonzero = solid: those nodes become
 * NODE_STRUCT (in addition to POISEUILLE's pipe wall), are never streamed or
 * collided and export as zeros; a FLUID node next to one takes half-way
 * bounce-back; donors outside the box keep the case's own rules.  NULL
 * removes the mask.  Restarts the domain from its initial state (as
 * lbm_initialize).  Not for batch members. */
int lbm_set_solid_mask(lbm_domain* d, const unsigned char* mask);

/* ---------------------------------------------------------------------
 * Convergence stop (kernel.cu:232-248 prints sum |PrevDen - CurrDen| every
 * 100 steps; here the same residual ends the run).
 *
 * Steps in chunks of check_every (>= 1) until the FP64 residual
 * sum |rho_k - rho_(k-1)| of the last step of a chunk is <= tol, or
 * max_steps have been taken.  *steps_taken (may be NULL) = steps of this
 * call, *residual (may be NULL) = the last residual measured.  The residual
 * check synchronises the stream once per chunk.  Returns LBM_OK whether or
 * not the tolerance was reached; compare *residual with tol.
 * --------------------------------------------------------------------- */
int lbm_run_until_converged(lbm_domain* d, int max_steps, int check_every, double tol,
                            int* steps_taken, double* residual);

/* ---------------------------------------------------------------------
 * Checkpoint / restart through the padded arF (the reference's restart
 * fields irestart / irst, struct.h:84, only name its output files).
 *
 * lbm_save_checkpoint writes a 64-byte header ("LBMCKPT1", nx, ny, nz, 19,
 * steps done, storage, casetype) and the ghost-padded AoS arF
 * [ny+2][nz+2][nx+2][19] as float32 (what lbm_export_arF(padded = 1)
 * returns).  lbm_load_checkpoint checks the extents and imports it as
 * lbm_import_arF does; the handle's step count restarts at 0 and *step (may
 * be NULL) receives the count stored in the file.  Continuing a cavity after
 * a load gives the same populations as never stopping.
 * --------------------------------------------------------------------- */
int lbm_save_checkpoint(lbm_domain* d, const char* path);
int lbm_load_checkpoint(lbm_domain* d, const char* path, long long* step);

/* ---------------------------------------------------------------------
 * Output files: saveFile (kernel.cu:699-1018).
 *
 * LBM_SAVE_VTU (BINARYTYPE, common.h:29): VTK XML UnstructuredGrid with
 *   appended raw data (UInt64 block headers): Float64 point coordinates,
 *   Int32 hexahedron connectivity / offsets, UInt8 types (12), Float64
 *   Velocity (3 components) and Density, Int32 flags Fluid, Fixed Wall,
 *   Moving Wall, Inlet, Outlet, Struct, in kernel.cu's order and names.
 *   Written as <dir>/Output%06d.vtu (kernel.cu:706 with SAVE_PATH = dir).
 * LBM_SAVE_CSV (CSVTYPE, common.h:30): <dir>/result.csv
 *   ("x,y,z,rho,u,v,w", one line per node in [y][z][x] order) and
 *   <dir>/section.csv ("y/Y,u": u_x*10 along y at x = z = 49), with
 *   kernel.cu's printf formats, byte for byte.
 * --------------------------------------------------------------------- */
enum { LBM_SAVE_VTU = 0, LBM_SAVE_CSV = 1 };

/* Host writers over caller arrays [ny][nz][nx] (no device involved).
 * lbm_write_csv: either path may be NULL to skip that file. */
int lbm_write_vtu(const char* path, int nx, int ny, int nz, const float* den, const float* velx,
                  const float* vely, const float* velz, const int* node_type);
int lbm_write_csv(const char* result_path, const char* section_path, int nx, int ny, int nz,
                  const float* den, const float* velx, const float* vely, const float* velz);

/* Capture the macroscopic state after the last step into a snapshot: a
 * device-side copy on the handle's stream, then an asynchronous copy to
 * pinned host memory on a side stream, so the next lbm_run_simulation can
 * start at once and overlaps the transfer.  The first call also reads the
 * node types (synchronously) and allocates the snapshot buffers. */
int lbm_snapshot(lbm_domain* d);

/* Write the last snapshot (waits for its host copy) as savetype into dir
 * (NULL = "./result/", as SAVE_PATH; created if its parent exists) with
 * file index `index`.  May run on
 * another host thread while that thread's partner keeps stepping the same
 * handle; it must not overlap an lbm_snapshot call on the handle. */
int lbm_save_snapshot(lbm_domain* d, int savetype, const char* dir, int index);

/* lbm_snapshot + lbm_save_snapshot. */
int lbm_save_file(lbm_domain* d, int savetype, const char* dir, int index);

/* No counterpart in the reference.  The diagnostics of lbm_diagnostics
 * (same 8 values, same order, FP64) over caller-owned device arrays of n
 * nodes, for callers that cannot allocate device memory when they need them:
 * a serving loop whose device memory is all handed to resident domains, code
 * that must not synchronise the device the way cudaMalloc/cudaFree may, or
 * fields whose memory belongs to another runtime.  It allocates nothing:
 * the per-block partial sums live in a file-scope __device__ array of the
 * library sized for at most 67,108,864 nodes (264 KB, held by every GPU that
 * loads the library until exit); larger n returns LBM_ERR_INVALID.
 * den_prev may be NULL (out[4] is then 0).  Work is ordered on `stream`
 * (a cudaStream_t, NULL = default stream); every call synchronises that
 * stream and copies the 8 results to the host before it returns.
 * Every call synchronises `stream`, so it cannot be made on a stream that
 * is being captured into a graph.  The first call on a device looks up the
 * array's device address (cudaGetSymbolAddress) and keeps it for later calls
 * on that device; do not use the function across a cudaDeviceReset of the
 * device (the kept address would be stale).  All calls on a device share the array and it keeps the last
 * call's contents: calls that overlap on the GPU race and must be
 * serialised by the caller. */
int lbm_field_diagnostics_static(const float* den, const float* den_prev, const float* velx,
                                 const float* vely, const float* velz, long long n,
                                 double out[8], void* stream);

/* Block until all work of the handle is done. */
int lbm_sync(lbm_domain* d);

/* Device bytes held by the handle. */
int lbm_device_bytes(const lbm_domain* d, size_t* bytes);

/* The device arrays of the macroscopic state after the last step, as the
 * reference's LBMSolver::m_DeviceNode exposes them (m_dCurrDen, m_dPrevDen,
 * m_dCurrVelx/y/z; struct.h:30-50): [ny][nz][nx] FP32 each, owned by the
 * handle, written by the handle's stream; valid until its next step,
 * import or destroy.  prev_den holds the density of the step before (0
 * right after initialize / import).  Any pointer may be NULL.  (The
 * populations are in the library's private layout; lbm_export_arF reads
 * them as the reference's arF.) */
int lbm_device_fields(lbm_domain* d, float** den, float** prev_den, float** velx, float** vely,
                      float** velz);

/* Bytes a domain of this case would hold (for admission control). */
int lbm_estimate_bytes(const Inputval* pinput, const lbm_options* opt,
                       size_t* bytes);

/* Average duration in milliseconds of the fused step kernel over the last
 * lbm_run_simulation call, measured with CUDA events on the handle's
 * stream around the kernel launches (synchronises). */
int lbm_last_run_ms(lbm_domain* d, float* ms);

/* ---------------------------------------------------------------------
 * Memory-pattern ceilings (no counterpart in the reference: a measurement
 * tool).  Times `iters` launches of a kernel that performs exactly the
 * global loads and stores of one lattice update of a step form (19 loads
 * and 19 stores per node, same addresses, access widths and thread
 * mapping) with a token amount of arithmetic, on an n^3 box (n a multiple
 * of 32, 32..512) of F32 or F16 storage, after 3 untimed launches.  No step
 * kernel with that memory pattern can be faster.  *mlups = updated nodes per
 * second / 1e6, *gbs = 2*19*bytes per node at that rate.  Allocates and
 * frees two lattices of 19*n^3 elements; synchronises the device work it
 * issued on its own stream.
 * --------------------------------------------------------------------- */
enum {
  LBM_PATTERN_COPY = 0,         /* 19 planes in, 19 out, at the node, 16-byte vectors */
  LBM_PATTERN_PULL = 1,         /* pull from x - c_q, one element per access   */
  LBM_PATTERN_PULL_PAIRED = 2,  /* 16-bit rows as words (w, w + px/2): 32-bit
                                   accesses, two nodes per thread              */
  LBM_PATTERN_AA_LOCAL = 3,     /* AA local step, one element per access       */
  LBM_PATTERN_AA_NEIGHBOR = 4,  /* AA neighbour step, one element per access   */
  LBM_PATTERN_AA_LOCAL_V8 = 5,  /* AA local step, 8-byte vectors per lane      */
  LBM_PATTERN_AA_LOCAL_V16 = 6, /* AA local step, 16-byte vectors per lane     */
  /* 16-bit only: */
  LBM_PATTERN_AA_PAIRED_LOCAL = 7,     /* AA steps over paired rows: 32-bit   */
  LBM_PATTERN_AA_PAIRED_NEIGHBOR = 8,  /* words, two nodes per thread         */
  LBM_PATTERN_PULL_QUAD = 9,           /* rows as 8-byte words of the nodes   */
  LBM_PATTERN_AA_QUAD_LOCAL = 10,      /* (w, w+Q, w+2Q, w+3Q), Q = px/4:     */
  LBM_PATTERN_AA_QUAD_NEIGHBOR = 11    /* four nodes per thread, x shifts are
                                          whole-word shifts                   */
};
int lbm_pattern_ceiling(int pattern, int storage, int n, int iters, double* mlups,
                        double* gbs);

/* ------------------------------------------------------------------ */
/* Batches: many independent domains of uneven size resident on one    */
/* GPU, stepped together by one persistent kernel per time step over a  */
/* tile work-list (every tile a run of nodes of one domain).  Steps are */
/* issued in chunks captured as CUDA graphs; each domain advances to    */
/* its own step target, so domains can join and leave between chunks   */
/* (continuous batching).  No reference counterpart: the reference runs */
/* one domain per program (main.cpp:287-291).                           */
/* ------------------------------------------------------------------ */
typedef struct lbm_batch lbm_batch;

typedef struct lbm_batch_options {
  int device;             /* CUDA device ordinal                              */
  size_t hbm_budget;      /* bytes of the device pool holding every domain    */
  int chunk_steps;        /* steps per captured graph chunk (even), 0 = 32    */
  int block;              /* threads per CTA (128 or 256), 0 = autotuned/256  */
  int nodes_per_thread;   /* nodes per lane per warp tile (1..16), 0 = 2      */
  int ctas_per_sm;        /* persistent CTAs per SM, 0 = max resident         */
  int schedule;           /* persistent kernel over warp tiles: 0 each warp a
                             contiguous range, 1 warp-stride; 2: flat grids,
                             members packed into sets whose arguments travel
                             as kernel parameters, one launch chain per set
                             in the chunk graph (block, nodes_per_thread,
                             ctas_per_sm and regs do not apply); default 2   */
  int regs;               /* kernel build: 0 = 64 registers, 1 = 80           */
  int own_set_ctas;       /* schedule 2: a member of at least this many CTAs
                             (of 128 nodes or paired words) is a set of its
                             own, stepped by its single-domain kernel;
                             0 = 2048                                          */
  int reserved[5];
} lbm_batch_options;

void lbm_batch_default_options(lbm_batch_options* bo);

/* Create a batch: reserves bo->hbm_budget bytes of device memory. */
int lbm_batch_create(const lbm_batch_options* bo, lbm_batch** out);
int lbm_batch_destroy(lbm_batch* b);

/* Admit a domain with a step target.  Its memory comes from the pool;
 * LBM_ERR_BUDGET when it does not fit.  The initial state is built on the
 * batch stream.  Storage LBM_STORE_F64 is not supported in batches. */
int lbm_batch_add(lbm_batch* b, const Inputval* pinput, const lbm_options* opt,
                  long long target_steps, int* id);

/* Issue `steps` more steps to every admitted domain that has not reached
 * its target (each stops at its own target).  Asynchronous. */
int lbm_batch_step(lbm_batch* b, int steps);

/* Ids (up to max) of domains that reached their target and whose last
 * chunk has completed on the GPU; non-blocking.  *n = count written. */
int lbm_batch_poll(lbm_batch* b, int* ids, int max, int* n);

/* The domain handle of a batch member: lbm_export_arF, lbm_get_macroscopic,
 * lbm_diagnostics and lbm_steps_done work on it (they synchronise the batch
 * stream).  Owned by the batch. */
int lbm_batch_domain(lbm_batch* b, int id, lbm_domain** d);

/* CurrDen / CurrVel* of a member that reached its target, [ny][nz][nx]
 * (any pointer may be NULL).  Waits only for the member's last chunk, so
 * the chunks queued behind it keep running. */
int lbm_batch_fetch(lbm_batch* b, int id, float* den, float* velx, float* vely, float* velz);

/* Release a member's memory back to the pool (waits for its last chunk). */
int lbm_batch_remove(lbm_batch* b, int id);

int lbm_batch_sync(lbm_batch* b);

/* Bytes of the pool in use, free (largest block), and domains resident. */
int lbm_batch_usage(lbm_batch* b, size_t* used, size_t* largest_free, int* ndomains);

/* Bytes a domain of this case takes from a batch pool. */
int lbm_batch_domain_bytes(const Inputval* pinput, const lbm_options* opt, size_t* bytes);

/* Project autotuner: run `trial_steps` real steps of the current batch with
 * each candidate (register build, schedule, block, nodes per thread, CTAs per
 * SM) and keep the fastest; writes the choice into *chosen (may be NULL).
 * The trials consume the members' steps: up to 13 candidates each run
 * `trial_steps` real steps, so up to 13 * trial_steps steps of every member
 * count toward its target (a member that reaches its target stops, as in
 * lbm_batch_step).  Tune on members whose targets leave room for this, or on
 * throwaway members of the same mix. */
int lbm_batch_autotune(lbm_batch* b, int trial_steps, lbm_batch_options* chosen);

/* Average milliseconds per step of the last lbm_batch_step call, measured
 * with CUDA events on the batch stream (synchronises); *lups = lattice
 * updates issued by that call. */
int lbm_batch_last_step_ms(lbm_batch* b, float* ms, long long* lups);

/* ------------------------------------------------------------------ */
/* Serving: a request queue over one batch.  A request is one solve (a  */
/* case, its options, a step budget and an optional residual            */
/* tolerance).  lbm_server_progress admits queued requests while their  */
/* state fits the pool (and the resident backlog stays under a horizon),*/
/* runs one chunk of steps for every resident request, and retires the  */
/* requests that reached their budget or whose density residual         */
/* sum |rho_k - rho_(k-1)| (the quantity kernel.cu:232-248 prints) fell */
/* to their tolerance at a check, copying rho and u to host memory and  */
/* returning their device memory to the pool.  No reference             */
/* counterpart: the reference runs one case per program.                */
/* ------------------------------------------------------------------ */
typedef struct lbm_server lbm_server;

enum {
  LBM_SERVE_FIFO = 0,     /* arrival order; a request that does not fit blocks
                             the ones behind it (no overtaking)               */
  LBM_SERVE_SHORTEST = 1  /* least work (nodes x steps) first; requests that
                             do not fit are skipped                           */
};

enum { LBM_REQ_QUEUED = 0, LBM_REQ_RESIDENT = 1, LBM_REQ_DONE = 2 };

typedef struct lbm_server_options {
  lbm_batch_options batch;  /* the batch under the queue (pool, chunk, ...)  */
  int policy;               /* LBM_SERVE_*                                    */
  int check_every;          /* steps between residual checks: a positive
                               multiple of the chunk, default 256              */
  double backlog_horizon_s; /* > 0: admit while the resident requests owe at
                               most this many seconds of work at
                               nominal_mlups; 0 = limited by the pool only    */
  double nominal_mlups;     /* the rate the horizon is measured in            */
  int reserved[6];
} lbm_server_options;

typedef struct lbm_server_request {
  int state;                /* LBM_REQ_*                                       */
  int converged;            /* 1: retired early at its residual tolerance      */
  long long steps_done;
  double residual;          /* last checked residual, -1 if never checked      */
  double t_arrive, t_admit, t_done;  /* seconds since the server was created,
                                        -1 where not reached                 */
} lbm_server_request;

typedef struct lbm_server_summary {
  long long submitted, admitted, completed, converged, queued, resident;
  double elapsed_s;                   /* since the server was created          */
  double tts_p50_s, tts_p99_s;        /* arrival -> result on the host         */
  double service_p50_s, service_p99_s;/* admission -> result on the host       */
  double executed_lups;               /* lattice updates run                    */
  double completed_lups;              /* ... by requests that completed         */
  double aggregate_mlups;             /* executed_lups / elapsed_s / 1e6        */
  size_t pool_used_bytes;
} lbm_server_summary;

void lbm_server_default_options(lbm_server_options* so);
int lbm_server_create(const lbm_server_options* so, lbm_server** out);
int lbm_server_destroy(lbm_server* s);

/* Queue a request; *id names it.  LBM_ERR_BUDGET when its state can never
 * fit the pool.  tol > 0 enables the residual check (domains of at most
 * 67,108,864 nodes); tol = 0 runs the full budget. */
int lbm_server_submit(lbm_server* s, const Inputval* pinput, const lbm_options* opt,
                      long long steps, double tol, int* id);

/* One turn of the loop: admit, one chunk, checks, retire.  *completed (may
 * be NULL) = requests that completed during the call. */
int lbm_server_progress(lbm_server* s, int* completed);

/* Turn the loop until request id is done. */
int lbm_server_wait(lbm_server* s, int id);

/* Status of a request, and (when done) its CurrDen / CurrVel* in
 * [ny][nz][nx]; any pointer may be NULL. */
int lbm_server_result(lbm_server* s, int id, float* den, float* velx, float* vely, float* velz,
                      lbm_server_request* info);

/* Forget a done request and free its host copy. */
int lbm_server_release(lbm_server* s, int id);

int lbm_server_stats(lbm_server* s, lbm_server_summary* st);

/* The batch under the queue (owned by the server). */
int lbm_server_batch(lbm_server* s, lbm_batch** b);

#ifdef __cplusplus
}
#endif
#endif /* LBM_B200_H */
