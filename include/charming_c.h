/* charming-b200 C ABI.
 *
 * Plain C entry points over the single-GPU runtime: plain pointers and sizes,
 * no CUDA or torch types. Every function returns an int status
 * (CHARMING_OK == 0) unless stated otherwise.
 *
 * The reference (minitu/charming) has no C ABI: its only host entry is the
 * process main() in src/charming.cu:50-263 that every example links, so
 * each entry point below names the part of that function (or of the example
 * programs) it replaces.
 */
#ifndef CHARMING_C_H_
#define CHARMING_C_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes (device error words and host failures) ---------------- */
enum {
  CHARMING_OK = 0,
  CHARMING_ERR_RING_FULL = 1,       /* no inbox space within the wait limit   */
  CHARMING_ERR_STASH_FULL = 2,      /* refnum stash out of descriptors/bytes  */
  CHARMING_ERR_BAD_TARGET = 3,      /* invalid chare array / index / entry    */
  CHARMING_ERR_BARRIER_TIMEOUT = 4, /* a PE did not reach a barrier in time   */
  CHARMING_ERR_IDLE_TIMEOUT = 5,    /* nothing delivered anywhere for too long*/
  CHARMING_ERR_DEADLINE = 6,        /* run exceeded its deadline              */
  CHARMING_ERR_BAD_MSG = 7,         /* malformed message in an inbox          */
  CHARMING_ERR_MSG_TOO_LARGE = 8,   /* message larger than max_msg_bytes      */
  CHARMING_ERR_HOST_STOP = 9,       /* stopped by the host                    */
  CHARMING_ERR_TOO_MANY_TYPES = 10, /* > CHARE_TYPE_CNT_MAX proxies on a PE   */
  CHARMING_ERR_TOO_MANY_EMS = 11,   /* > EM_CNT_MAX entry methods             */
  CHARMING_ERR_PIPELINE = 12,       /* bulk-copy pipeline wait ran out        */
  CHARMING_ERR_LAUNCH = 13,         /* scheduler launch failed                */
  CHARMING_ERR_CONFIG = 14,         /* invalid configuration or argument      */
  CHARMING_ERR_CUDA = 15,           /* CUDA runtime error (see last_error)    */
  CHARMING_ERR_NOT_INIT = 16,       /* charming_init() not called             */
  CHARMING_ERR_NO_MEMORY = 17,      /* allocation or HBM budget exhausted     */
  CHARMING_ERR_APP = 18,            /* built-in program reported a failure    */
  CHARMING_ERR_TOO_MANY_WAITS = 19  /* > ASYNC_WAIT_MAX pending async_waits    */
};

/* ---- runtime ------------------------------------------------------------ */

/* Runtime configuration. Replaces the constants and limits fixed in the
 * reference's main (src/charming.cu:85-100 topology, :197-203 limits,
 * :207-209 grid) and transport (src/comm/get/get.cu:20-32 buffer sizes). */
typedef struct charming_config {
  int device;               /* CUDA device ordinal                           */
  int pes_per_sm;           /* PE thread blocks per SM (1 or 2)              */
  int threads_per_pe;       /* threads per PE block, multiple of 32, <= 512  */
  int n_pes;                /* 0: SMs * pes_per_sm                           */
  uint64_t ring_bytes;      /* inbox ring bytes per PE (power of two)        */
  uint64_t max_msg_bytes;   /* largest message incl. 32-byte header          */
  uint64_t stash_bytes;     /* refnum stash arena bytes per PE               */
  int stash_entries;        /* refnum stash descriptors per PE               */
  uint64_t heap_bytes;      /* device malloc heap (chare objects)            */
  uint64_t stack_bytes;     /* per-thread stack                              */
  double deadline_s;        /* hard limit on one scheduler run               */
  double idle_timeout_s;    /* stop if no message is delivered for this long */
  int free_chares_at_exit;  /* delete proxies/chares when a run ends         */
  int verbose;              /* print the configuration (PINFO) on init       */
  int gpu_level;            /* 1: GPU-level mode, the reference's default
                               build (src/sched/scheduler.cu:240-333): all
                               blocks (n_pes of them, 0: one per SM slot)
                               form a single PE that runs every entry method
                               and collective send together; n_pes() is 1.
                               0: SM-level mode, one PE per block          */
} charming_config;

/* Fills *cfg with defaults (148 PEs on a B200, 512 threads, 4 MiB rings). */
void charming_default_config(charming_config* cfg);

/* Device setup, buffer allocation, constants. Replaces src/charming.cu:50-231
 * (NVSHMEM/MPI init, proxy tables, limits, comm_init_host). */
int charming_init(const charming_config* cfg);

/* ---- several GPUs ----------------------------------------------------------
 * One process per GPU of one NVSwitch domain. Replaces the reference's
 * multi-GPU transport: NVSHMEM PEs, with a communication element (CE) per
 * GPU that relays messages to and from other GPUs as request/forward
 * messages (src/comm/get/get.cu:518-690, :783-862; src/sched/scheduler.cu:
 * 78-163). Here every GPU's inbox side is exported with CUDA IPC and mapped
 * by the others, and a PE sends to a PE on another GPU exactly as to one on
 * its own GPU: its ticket atomic and payload stores cross NVLink. There is
 * no CE. PEs are numbered globally: GPU g holds PEs g*P .. g*P + P - 1, P
 * (PEs per GPU) equal on all GPUs; charm::n_pes() counts all of them.
 *
 * The host supplies two collectives over the processes (torch.distributed
 * in the Python package, files in a shared directory in the process main):
 * allgather of `bytes` from each rank into all[world * bytes] in rank order,
 * and a barrier. Each returns 0 on success. */
typedef int (*charming_allgather_fn)(void* ctx, const void* mine, void* all, size_t bytes);
typedef int (*charming_barrier_fn)(void* ctx);

typedef struct charming_devices {
  int rank;                  /* this process's GPU in the run, 0..world-1    */
  int world;                 /* processes (GPUs) of the run; 1: this GPU only */
  int virtual_devs;          /* > 1, with world == 1: this GPU's PEs form that
                                many GPUs, each with its own inbox memory and
                                control words, in one launch (the multi-GPU
                                transport's code path, run on one GPU)      */
  int reserved;
  charming_allgather_fn allgather;
  charming_barrier_fn barrier;
  void* ctx;                 /* passed to both                              */
} charming_devices;

/* charming_init over several GPUs (devs == NULL, or world == 1 and
 * virtual_devs <= 1: charming_init). With world > 1 it is collective: every
 * rank calls it with equal PEs per GPU, ring and message sizes, and
 * charming_run and charming_fini are collective too. SM-level mode only;
 * the message programs (hello, refnum, pingpong, fan-out) and programs
 * linked against the process main run over several processes. */
int charming_init_devices(const charming_config* cfg, const charming_devices* devs);

/* Runs charm::main on every PE and then the scheduler until charm::end(),
 * an error, or a limit. One cooperative launch of the persistent scheduler
 * kernel. Replaces src/charming.cu:146-169 (argv to device) and :234-244
 * (collective launch + sync). */
int charming_run(int argc, char** argv);

/* Releases everything charming_init allocated (src/charming.cu:250-261). */
int charming_fini(void);

/* Device time over several runs: CUDA events on the runtime's stream around
 * everything enqueued between start and stop (the reference times with
 * device-side clocks inside entry methods, examples/jacobi2d/jacobi2d.cu:
 * 236-262). */
int charming_timer_start(void);
int charming_timer_stop(double* ms);

/* Effective configuration after init (n_pes, threads, smem bytes). */
typedef struct charming_info {
  int n_pes;
  int n_sms;
  int threads_per_pe;
  int smem_bytes_per_pe;     /* dynamic shared memory per PE block       */
  int smem_scratch_bytes;    /* of which available to entry methods      */
  int regs_per_thread;       /* of the scheduler kernel                  */
  uint64_t ring_bytes;
  uint64_t max_msg_bytes;    /* largest message incl. 32-byte header     */
  uint64_t device_bytes;     /* runtime buffers on the device            */
  uint64_t stack_bytes;      /* per-thread stack limit in effect         */
  uint64_t local_bytes;      /* scheduler kernel's static local memory   */
  int n_blocks;              /* thread blocks of the scheduler launch    */
  int gpu_level;             /* 1: GPU-level mode (n_pes is 1)           */
  int n_devs;                /* GPUs of the run (virtual ones included)  */
  int my_dev;                /* this process's (first) GPU               */
} charming_info;
int charming_get_info(charming_info* out);

/* Statistics of the last run, summed over PEs. */
typedef struct charming_stats {
  uint64_t delivered;        /* entry methods run                        */
  uint64_t sent;             /* messages sent                            */
  uint64_t stashed;          /* messages parked on refnum mismatch       */
  uint64_t revived;          /* parked messages made deliverable         */
  uint64_t bytes_sent;       /* payload bytes                            */
  uint64_t idle_polls;       /* empty inbox polls                        */
  uint64_t space_waits;      /* sends that waited for ring space         */
  double kernel_ms;          /* CUDA-event time of the scheduler launch  */
  double loop_ms;            /* first loop start to last loop end        */
  double main_ms;            /* max over PEs: kernel start to loop start
                                (charm::main, chare creation, barriers)  */
  int status;                /* status code of the run                   */
  int err_pe, err_info0, err_info1;
  double idle_ms;            /* mean over PEs: time waiting on an empty
                                inbox (SM cycles at the nominal clock)   */
  double em_ms;              /* mean over PEs: time inside entry methods
                                (SM cycles at the nominal clock)         */
  uint64_t deferred;         /* sends moved to the sender's outbox because
                                the destination ring stayed full         */
  double ticket_ms;          /* mean over PEs: reserving thread waiting for
                                its inbox-ticket atomics (this and the
                                next: profiling builds only, else 0)     */
  double space_ms;           /* mean over PEs: then for ring space (a stale
                                head cache refreshed, or a full ring)    */
  uint64_t batched;          /* deliveries run beside others, one per warp,
                                in batches of warp-level entry methods   */
} charming_stats;
int charming_last_stats(charming_stats* out);

/* Message for a status code (static string). */
const char* charming_status_string(int code);
/* Last host-side CUDA error text (static buffer, may be empty). */
const char* charming_last_error(void);

/* ---- built-in programs (libcharming_b200.so) ---------------------------- */
enum { CHARMING_F64 = 0, CHARMING_F32 = 1 };

/* One Dirichlet problem on an (ny+2) x (nx+2) grid whose outer ring holds
 * fixed boundary values. Replaces the parameters of the reference's
 * examples/jacobi2d/jacobi2d.cu:26-85 (grid size, chare count, iterations). */
typedef struct charming_jacobi_problem {
  int nx, ny;          /* interior columns, rows                            */
  int px, py;          /* chares along x (columns) and y (rows); 0: auto    */
  int max_sweeps;      /* sweeps to run (cap when tol > 0)                  */
  int check_every;     /* residual check period in sweeps (0: none)         */
  double tol;          /* stop when ||r_k|| / ||r_0|| <= tol (0: never)      */
  double bc[4];        /* boundary values: top, bottom, left, right         */
} charming_jacobi_problem;

typedef struct charming_jacobi_options {
  int dtype;           /* CHARMING_F64, or CHARMING_F32 sweeps with an FP64
                          residual                                          */
  int chare_side;      /* auto decomposition: target chare side (0: 256)    */
  int tile_w;          /* sweep tile width in elements (0: default)         */
  int pipeline;        /* 1: TMA bulk-copy row pipeline, 0: direct loads    */
  int use_graph;       /* 1: replay each run from a captured CUDA graph     */
  int balance;         /* 1: place chares by work (greedy), 0: block map    */
  int halo_mode;       /* 0: halos land in the ghost ring of the sweep they
                          belong to (parity buffers); 1: halos carry refnum
                          = exchange and early ones wait in the stash       */
  int depth;           /* sweeps per halo exchange, 1..8, with ghost zones of
                          that depth (corners from diagonal neighbours when
                          > 1); 0: 6 for the direct sweep (with a residual
                          period K, the balanced split of K into passes of
                          at most 6: 5 for K = 10), 1 for the TMA pipeline;
                          capped by the smallest chare side.
                          The reference exchanges halos every sweep (1)     */
} charming_jacobi_options;

typedef struct charming_jacobi_result {
  int sweeps;          /* sweeps performed                                  */
  int checks;          /* residual checks performed                         */
  double res0;         /* ||S(u_0) - u_0||_2 (FP64)                          */
  double res_last;     /* last checked residual norm                        */
} charming_jacobi_result;

typedef struct charming_jacobi_info {
  int n_problems;
  int n_chares;
  int max_chares_per_pe;
  uint64_t interior_points;   /* sum of nx*ny                              */
  uint64_t grid_bytes;        /* device bytes of all chare grids           */
  uint64_t halo_msgs_per_sweep; /* halo messages per exchange (every `depth` sweeps) */
  double last_run_ms;         /* CUDA-event time of the last run           */
  /* the phase times below: SM cycles at the nominal clock */
  double sweep_ms_max;        /* last run: max over PEs of time in sweeps  */
  double sweep_ms_mean;       /* last run: mean over busy PEs              */
  double send_ms_mean;        /* last run: mean time packing/sending halos */
  double halo_ms_mean;        /* last run: mean time in halo entry methods */
  /* the next three: builds with -DCHARMING_PROFILE only (else 0) */
  double send_reserve_ms_mean;  /* of send_ms_mean: taking the ring space    */
  double send_publish_ms_mean;  /* of send_ms_mean: publishing the messages  */
  double send_setup_ms_mean;    /* of send_reserve_ms_mean: before the
                                   reservation call                         */
} charming_jacobi_info;

/* Decomposes the problems into chares (reference decomposition:
 * examples/jacobi2d/jacobi2d.cu:37-65) and allocates their grids. */
int charming_jacobi2d_create(const charming_jacobi_problem* probs, int n,
    const charming_jacobi_options* opt, void** handle);
/* Device-side initial state: boundary ring from bc[], interior 0. */
int charming_jacobi2d_init(void* handle);
/* Host grid ((ny+2)*(nx+2) values of the problem's dtype, row-major with the
 * boundary ring) -> chare blocks on the device. */
int charming_jacobi2d_load(void* handle, int prob, const void* host_grid);
/* Runs every problem to completion in one persistent scheduler launch. The
 * chare logic follows examples/jacobi2d/jacobi2d.cu:93-279 with halos tagged
 * refnum = sweep. */
int charming_jacobi2d_run(void* handle);
/* n_runs runs of charming_jacobi2d_run enqueued back to back on the
 * runtime's stream and synchronised once: no host work between them (a
 * status latch after each keeps the first failure, which is returned).
 * *total_ms: CUDA-event time of all of them; the statistics are the last
 * run's, last_run_ms their mean. */
int charming_jacobi2d_run_n(void* handle, int n_runs, double* total_ms);
/* Chare blocks -> host grid (same layout as load). */
int charming_jacobi2d_store(void* handle, int prob, void* host_grid);
int charming_jacobi2d_result(void* handle, int prob, charming_jacobi_result* out);
/* n solves of problem prob: host_in[k] (as load takes it) -> host_out[k] (as
 * store gives it), each exactly load + run + store, pipelined: the copies of
 * solve k+1's input and of solve k-1's result run on their own streams while
 * solve k runs (two device staging buffers each way). Host buffers should be
 * pinned for the copies to overlap. *out_ms: time from the first input copy
 * to the last result copy. Replaces a host loop over the reference's
 * process main (src/charming.cu:50-263) with the grid moved in and out. */
int charming_jacobi2d_solve_stream(void* handle, int prob, int n, const void* const* host_in,
    void* const* host_out, double* out_ms);
int charming_jacobi2d_get_info(void* handle, charming_jacobi_info* out);
int charming_jacobi2d_destroy(void* handle);

/* Sweeps one grid without allocating device memory (no counterpart in the
 * reference). For callers that must not allocate: code that serves this
 * library device buffers from its own pool and forbids other allocations,
 * or that cannot afford the device synchronisation a cudaMalloc implies.
 * dev_in and dev_out are device grids of (ny+2)*(nx+2) values of dtype,
 * row-major with the boundary ring, not overlapping; dev_out receives the
 * grid after `sweeps` sweeps, equal bit for bit to charming_jacobi2d_run's
 * result with max_sweeps = sweeps and check_every = 0. The second grid
 * lives in a 16 MiB scratch array inside the library (one per GPU, held
 * until exit), so (nx+2)*(ny+2)*element size must be <= 16 MiB, else
 * CHARMING_ERR_CONFIG; so are pointers not aligned to the element size.
 * Works on the current device and the legacy default stream and returns
 * when done (it synchronises that stream), so it must not be called while
 * any stream capture is in progress. The first call on a device also looks
 * up the scratch's device address and the device's multiprocessor count.
 * All calls share the scratch: calls that overlap on the GPU race. */
int charming_jacobi2d_sweeps_noalloc(int dtype, int nx, int ny, int sweeps,
    const void* dev_in, void* dev_out);

/* 3-D Jacobi sweeps (the 7-point FP64 stencil of examples/jacobi-kernel/
 * jacobi_kernel.cu:36-48, multiplied by its literal 0.142857): grid is the
 * host's (nz+2) x (ny+2) x (nx+2) doubles, x fastest, shell fixed; it
 * receives the result of `sweeps` sweeps. *out_ms: device time of the
 * sweeps (copies excluded). */
int charming_jacobi3d(int nx, int ny, int nz, int sweeps, double* grid, double* out_ms);

/* Jacobi2d over a 1-D row decomposition (examples/jacobi2d-decomp1d/
 * jacobi2d.cu): an ny x nx FP32 grid (nx a multiple of 4) split into bands
 * of rows over n_chares chares as its Block::init does (:144-198), periodic
 * top/bottom neighbours, columns 0 and nx-1 fixed to sin(2*PI*(g-1)/(ny-3))
 * per global row g, the 4-point stencil of its jacobi_kernel (:374-383) for
 * `iters` iterations. mode 0: boundary rows written into the neighbours'
 * buffers and signalled, waited for inside the entry method (one chare per
 * PE); 1: the same, resumed by async_wait; 2: boundary rows as messages
 * tagged with the iteration as refnum. host_out receives the bands' rows
 * ((ny-2) x nx floats); *out_ms the scheduler loop's time. */
int charming_jacobi2d_decomp1d(int n_chares, int nx, int ny, int iters, int mode, float* host_out,
    double* out_ms);

/* SM-to-SM pingpong floor: two thread blocks on different SMs bounce a
 * counter round_trips times, without the runtime (replaces the reference's
 * raw baseline, examples/baseline/baseline.cu:14-160, which prints the time
 * per iteration). mode 0: release store / acquire poll by one thread per
 * block (the floor); 1: relaxed polls plus one acquire fence per hit; 2:
 * mode 0 with a block barrier on each side of every hop; 3: the reference's
 * scheme (4 slots per SM pair, block-wide slot scans, atomicCAS publish and
 * clear). One-way time = round-trip time / 2 (block 0's clock). sm_pair
 * (optional) receives the two blocks' SM ids. */
int charming_sm_pingpong(int mode, int round_trips, double* oneway_ns, double* oneway_cycles,
    int* sm_pair);

/* Sweep throughput without messages (no reference counterpart; it times
 * the chare sweep of examples/jacobi2d/jacobi2d.cu:327-334 as implemented
 * here): n_blocks (<= n_pes) PE-shaped thread blocks each run `passes`
 * passes of `depth` sweeps over their own w x h chare block. variant 0:
 * multi-sweep pass with phase-split items, 1: with single-loop items
 * (depth >= 2), 2: one
 * direct sweep per pass (depth 1). *ms receives the kernel time. */
int charming_sweep_bench(int dtype, int w, int h, int depth, int passes, int n_blocks, int variant,
    double* ms);

/* async_wait chain (reference include/chare.h:214-239, src/comm/get/get.cu:
 * 1172-1202): chare i's entry method runs once its two signal words are >= 1,
 * which chare i-1 sets from its own; the host sets chare 0's. order[i]
 * receives chare i's wake position (-1: never woke). broken = 1: nobody
 * signals the last chare, so the run ends at the idle timeout
 * (CHARMING_ERR_IDLE_TIMEOUT). */
int charming_async_wait_chain(int n_chares, int broken, int* order, int n_order);

/* malloc_user / free_user check (reference include/charming.h:33-34,
 * src/comm/get/get.cu:1348-1362): each of n_chares takes `rounds` rounds of
 * blocks_per_round (<= 16) seeded-size blocks from its PE's heap, fills and
 * checks them, frees them out of order, then hands one block to the next
 * chare, which checks it on its PE. counters[0..6]: blocks taken, pattern
 * errors, allocation failures, blocks checked by another chare, blocks
 * freed, chares done, bytes taken. */
int charming_user_heap_check(int n_chares, int blocks_per_round, int rounds, uint64_t seed,
    uint64_t* counters);

/* 1-D Jacobi chares (examples/jacobi1d/jacobi1d.cu:62-170): n_chares blocks
 * of `width` points, 5-point window sum/5, boundary 10 and interior 0 as in
 * that example; result is the (n_chares*width + 4)-point array. */
int charming_jacobi1d(int n_chares, int width, int sweeps, double* host_out,
    double* out_ms);

/* Pingpong between chares on PEs 0 and n_pes/2 (examples/pingpong/
 * pingpong.cu:17-217). Payload bytes are a seeded SplitMix64 stream; with
 * verify=1 every received payload is checksummed and compared. */
typedef struct charming_pingpong_result {
  uint64_t size;
  double oneway_us;          /* mean one-way latency                     */
  double oneway_cycles;      /* same, in SM clock cycles                 */
  uint64_t checksum_errors;
} charming_pingpong_result;
int charming_pingpong(const uint64_t* sizes, int n_sizes, int round_trips,
    int warmup, uint64_t seed, int verify, charming_pingpong_result* out,
    int* sm_pair);

/* Fan-out: n_chares chares each send msgs_per_chare messages of payload_bytes
 * to seeded destinations. mode 0: refnum -1 (plain FIFO); mode 1: message k
 * carries refnum k and receivers advance their refnum after the expected
 * count. log receives one record per delivery: {dst, src, k, refnum,
 * seq_at_dst, checksum_lo, checksum_hi, pad} (8 x uint32). */
int charming_fanout(int n_chares, int msgs_per_chare, int payload_bytes,
    uint64_t seed, int mode, uint32_t* log, uint64_t log_capacity,
    uint64_t* n_logged, double* out_ms);

/* Hello chain (examples/hello/hello.cu): 2*n_pes chares pass an int along;
 * out[i] = value received by chare i. */
int charming_hello(int* out, int n_out, int* n_chares);

/* Refnum scenario (examples/refnum/refnum.cu:27-53, made to terminate):
 * out receives the refnums in the order chare 1 delivered them. */
int charming_refnum(int* out, int n_out, int* n_delivered);
/* Same with the two sends swapped: the refnum-0 message arrives first and is
 * parked in the stash until chare 1 moves to refnum 0. Expected out: 1, 0. */
int charming_refnum_reversed(int* out, int n_out, int* n_delivered);

/* ---- serving ------------------------------------------------------------ */
/* A solve server (no counterpart in the reference; it extends the reference's
 * model of chares in one persistent launch, src/sched/scheduler.cu:183-234,
 * to requests that arrive while the launch runs). charming_serve_start
 * launches the scheduler once with a pool of n_pes * workers_per_pe Jacobi2d
 * worker chares and a server chare on PE 0, and returns at once. Requests
 * (charming_jacobi_problem: size, boundary, sweep cap, residual period and
 * tolerance; px/py ignored, chares of chare_side) are admitted in arrival
 * order as a request slot, enough free workers and grid memory within the
 * HBM budget are available; admitted requests share the PEs with those
 * already running. A completed request's grid stays in HBM until
 * charming_serve_release; charming_serve_fetch copies it out ((ny+2)*(nx+2)
 * values of dtype with the boundary ring) while the server keeps running.
 * Results equal charming_jacobi2d_run's for the same problem and chare side
 * bit for bit. While a server runs it holds every PE: no other program of
 * this library may run, and the caller must not synchronise the whole
 * device. Call the serve functions from one host thread. */
typedef struct charming_serve_config {
  uint64_t hbm_budget_bytes; /* grids admitted at once must fit in this    */
  int max_inflight;          /* device problem slots                       */
  int workers_per_pe;        /* solver chares per PE                       */
  int chare_side;            /* requests are cut into chares of this side
                                (0: 2048)                                 */
  int dtype;                 /* CHARMING_F32 (FP64 residual) or F64        */
  double deadline_s;         /* server lifetime limit                      */
} charming_serve_config;

typedef struct charming_serve_completion {
  uint64_t tag;
  int status;
  int sweeps;
  double res0, res_last;
  double submit_s, admit_s, done_s;   /* host clock (seconds)             */
} charming_serve_completion;

typedef struct charming_serve_stats {
  uint64_t submitted, admitted, completed;
  uint64_t peak_bytes;
  int peak_inflight;
  double busy_s;
} charming_serve_stats;

int charming_serve_start(const charming_serve_config* cfg, void** server);
/* Queues a request under a caller-chosen tag (unique among requests not yet
 * released) and admits what fits; CHARMING_ERR_CONFIG for a request that could
 * never be admitted (larger than the budget or the worker pool). */
int charming_serve_submit(void* server, const charming_jacobi_problem* req,
    uint64_t tag);
/* Reads up to max_n completions (their slots and workers become free) and
 * admits what now fits; returns the run's status if the launch ended. */
int charming_serve_poll(void* server, charming_serve_completion* out,
    int max_n, int* n_out);
int charming_serve_fetch(void* server, uint64_t tag, void* host_grid);
/* Frees a completed request's grid memory. */
int charming_serve_release(void* server, uint64_t tag);
/* Stops admitting, waits for the requests in flight (within deadline_s),
 * ends the launch and frees everything; never-admitted requests are
 * dropped. */
int charming_serve_stop(void* server, charming_serve_stats* stats);

#ifdef __cplusplus
}
#endif

#endif /* CHARMING_C_H_ */
