// Host-side runtime internals shared by the C ABI implementations.
#pragma once

#include <cuda_runtime.h>
#include <string>
#include "rt.cuh"

namespace charm_host {

// Records `what` + the CUDA error text as the last error; returns
// CHARMING_ERR_CUDA when e != cudaSuccess, else CHARMING_OK.
int cuda_fail(cudaError_t e, const char* what);
void set_error_text(const std::string& s);

// charming_init() with defaults when nothing is initialised yet.
int ensure_init();
bool initialised();

cudaStream_t stream();
const charming_info& info();
// Processes of the run (1 unless charming_init_devices was given world > 1).
int n_procs();

// One scheduler run: reset kernel + cooperative launch on stream(), then
// synchronise and collect status and statistics.
int run_scheduler(int argc, char** argv);

// Enqueue reset + launch on `s` without synchronising (used for CUDA graph
// capture). argv is not forwarded (argc = 0).
int enqueue_scheduler(cudaStream_t s);

// After the work enqueued by enqueue_scheduler completed: read status and
// statistics into the last-run record; returns the run status.
int collect_run(double kernel_ms);
// Enqueues, after a scheduler run on s, a copy of the run's status words
// into latch[4] if latch[0] is still 0 (the first failing run of a series
// is kept; reading the latch needs no synchronisation per run).
int enqueue_status_latch(int* latch, cudaStream_t s);

// Run deadline of the following launches in seconds (<= 0: the configured
// one). Call only while no scheduler launch is running.
int set_deadline(double seconds);

// Sets the mapped host stop word read by the running scheduler
// (1 = stop normally, 2 = stop with CHARMING_ERR_HOST_STOP).
void request_stop(int value);

}  // namespace charm_host
