/* CPU baseline of the messaging microbenchmarks: test infrastructure,
 * timed beside the GPU numbers, never part of the product.
 *
 * The same workloads as the GPU's fan-out and pingpong programs
 * (charming_b200/csrc/apps/msgbench.cu), restated for host threads with
 * OpenMP: every thread owns one MPSC inbox ring (one ticket per message from
 * an atomic tail, a per-slot sequence word published with a release store,
 * so each (sender, receiver) pair stays FIFO, as on the GPU). Chares are
 * placed on threads by the reference's block rule (include/chare.h:136-176:
 * n / T per thread, the first n % T threads get one more).
 *
 *   fan-out: chare s sends message k (payload bytes from the seeded word
 *            stream) to chare mix64(seed ^ ((s*msgs+k+1)*G)) % n (refnum -1:
 *            the FIFO mode); receivers checksum every payload.
 *   pingpong: two threads bounce a payload of each size, round_trips times.
 */
#include <omp.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
static inline uint64_t gen_word(uint64_t seed, uint64_t stream, uint64_t j) {
  return mix64(seed ^ (stream * 0xD1B54A32D192ED03ULL) ^ (j * 0x9E3779B97F4A7C15ULL));
}

#define SLOT_WORDS 17 /* seq + up to 128 payload bytes */
#define MAX_PAYLOAD 128

typedef struct {
  _Atomic uint64_t seq;
  uint64_t w[SLOT_WORDS - 1];
} slot_t;

typedef struct {
  _Alignas(128) _Atomic uint64_t tail;
  _Alignas(128) _Atomic uint64_t head;
  slot_t* slots;
  uint64_t cap;
} inbox_t;

static int owner_of(int chare, int n, int T) {
  int per = n / T, rem = n % T;
  int big = rem * (per + 1);
  return chare < big ? chare / (per + 1) : rem + (chare - big) / (per > 0 ? per : 1);
}

/* Drains whatever is published in inbox `ib`; returns messages taken. */
static int drain(inbox_t* ib, int payload, uint64_t* csum) {
  int got = 0;
  uint64_t h = atomic_load_explicit(&ib->head, memory_order_relaxed);
  for (;;) {
    slot_t* s = &ib->slots[h % ib->cap];
    if (atomic_load_explicit(&s->seq, memory_order_acquire) != h + 1) break;
    int nw = (payload + 7) / 8;
    uint64_t c = 0;
    for (int j = 0; j < nw; j++) c += mix64(s->w[j] ^ (uint64_t)(j + 1));
    *csum += c;
    h++;
    got++;
    atomic_store_explicit(&ib->head, h, memory_order_release);
  }
  return got;
}

/* Fan-out of n chares x msgs messages of `payload` bytes on `threads`
 * threads. Returns the seconds of the parallel exchange; *delivered and
 * *checksum receive the totals. */
double cpu_fanout(int n, int msgs, int payload, uint64_t seed, int threads, uint64_t* delivered,
                  uint64_t* checksum) {
  if (payload > MAX_PAYLOAD || n <= 0 || msgs <= 0 || threads <= 0) return -1.0;
  const int T = threads;
  inbox_t* ib = aligned_alloc(128, sizeof(inbox_t) * (size_t)T);
  int* expect = calloc((size_t)T, sizeof(int));
  const uint64_t cap = 1u << 12;
  for (int t = 0; t < T; t++) {
    atomic_init(&ib[t].tail, 0);
    atomic_init(&ib[t].head, 0);
    ib[t].cap = cap;
    ib[t].slots = aligned_alloc(64, sizeof(slot_t) * cap);
    for (uint64_t i = 0; i < cap; i++) atomic_init(&ib[t].slots[i].seq, 0);
  }
  for (long long s = 0; s < n; s++)
    for (long long k = 0; k < msgs; k++) {
      uint64_t id = (uint64_t)(s * msgs + k);
      int dst = (int)(mix64(seed ^ ((id + 1) * 0x9E3779B97F4A7C15ULL)) % (uint64_t)n);
      expect[owner_of(dst, n, T)]++;
    }
  uint64_t total_got = 0, total_sum = 0;
  double t0 = 0, t1 = 0;
#pragma omp parallel num_threads(T) reduction(+ : total_got, total_sum)
  {
    const int me = omp_get_thread_num();
#pragma omp barrier
#pragma omp master
    t0 = omp_get_wtime();
#pragma omp barrier
    int per = n / T, rem = n % T;
    int c0 = me * per + (me < rem ? me : rem), c1 = c0 + per + (me < rem ? 1 : 0);
    int got = 0;
    uint64_t sum = 0;
    const int nw = (payload + 7) / 8;
    for (int s = c0; s < c1; s++) {
      for (int k = 0; k < msgs; k++) {
        uint64_t id = (uint64_t)s * (uint64_t)msgs + (uint64_t)k;
        int dst = (int)(mix64(seed ^ ((id + 1) * 0x9E3779B97F4A7C15ULL)) % (uint64_t)n);
        inbox_t* q = &ib[owner_of(dst, n, T)];
        uint64_t tk = atomic_fetch_add_explicit(&q->tail, 1, memory_order_relaxed);
        while (tk - atomic_load_explicit(&q->head, memory_order_acquire) >= q->cap)
          got += drain(&ib[me], payload, &sum);  /* keep receiving while the ring is full */
        slot_t* sl = &q->slots[tk % q->cap];
        for (int j = 0; j < nw; j++) {
          uint64_t w = gen_word(seed, id, (uint64_t)j);
          if (j == 0) w = (uint64_t)(uint32_t)s | ((uint64_t)(uint32_t)k << 32);
          if (j == 1) w = (uint64_t)(uint32_t)-1;
          sl->w[j] = w;
        }
        atomic_store_explicit(&sl->seq, tk + 1, memory_order_release);
        got += drain(&ib[me], payload, &sum);
      }
    }
    while (got < expect[me]) got += drain(&ib[me], payload, &sum);
#pragma omp barrier
#pragma omp master
    t1 = omp_get_wtime();
    total_got += (uint64_t)got;
    total_sum += sum;
  }
  for (int t = 0; t < T; t++) free(ib[t].slots);
  free(ib);
  free(expect);
  *delivered = total_got;
  *checksum = total_sum;
  return t1 - t0;
}

/* One-way latency (seconds) of a payload of `bytes` bounced between two
 * threads `round_trips` times, each side reading the whole payload. */
double cpu_pingpong(uint64_t bytes, int round_trips, uint64_t seed) {
  unsigned char* a = aligned_alloc(64, (bytes + 63) / 64 * 64);
  unsigned char* b = aligned_alloc(64, (bytes + 63) / 64 * 64);
  for (uint64_t i = 0; i < bytes; i++) a[i] = (unsigned char)gen_word(seed, 0, i / 8);
  _Alignas(128) _Atomic uint64_t fa = 0;
  _Alignas(128) _Atomic uint64_t fb = 0;
  double t0 = 0, t1 = 0;
  volatile uint64_t sink = 0;
#pragma omp parallel num_threads(2)
  {
    const int me = omp_get_thread_num();
#pragma omp barrier
    if (me == 0) t0 = omp_get_wtime();
    for (int r = 0; r < round_trips; r++) {
      if (me == 0) {
        atomic_store_explicit(&fa, (uint64_t)r + 1, memory_order_release);
        while (atomic_load_explicit(&fb, memory_order_acquire) != (uint64_t)r + 1) {
        }
        uint64_t c = 0;
        for (uint64_t i = 0; i < bytes; i += 8) c += b[i];
        sink += c;
      } else {
        while (atomic_load_explicit(&fa, memory_order_acquire) != (uint64_t)r + 1) {
        }
        memcpy(b, a, bytes);  /* receive and answer with the same bytes */
        atomic_store_explicit(&fb, (uint64_t)r + 1, memory_order_release);
      }
    }
    if (me == 0) t1 = omp_get_wtime();
  }
  (void)sink;
  free(a);
  free(b);
  return (t1 - t0) / (2.0 * round_trips);
}
