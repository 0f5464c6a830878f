// Run-time compiled kernels: CUDA source generated for one fused pass is
// compiled by NVRTC for sm_100a and loaded with the driver API, per device.
// NVRTC and the driver library are opened with dlopen on first use, so
// libqsim.so itself links against neither (it loads on hosts without a GPU).
#pragma once

#include <cstddef>
#include <cstdint>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace qs {
namespace jit {

// QS_JIT_OFF / QS_JIT_ASYNC / QS_JIT_SYNC (include/qsim.h)
int mode();
void set_mode(int m);

// Kernel `name` of `src`, loaded on the current device: non-null when ready.
// A source seen for the first time is queued for compilation on the pool
// (mode ASYNC: the call returns null until it is done) or compiled before
// returning (mode SYNC, or `block`).  Null when compilation failed; the
// first failure's log is kept for qs_jit_last_log.
// `load`: allow loading the cubin on this device now (false during stream
// capture: then only an already loaded kernel is returned).  *occ <- resident
// blocks per SM at `threads` threads and `smem` dynamic shared memory
// (computed when the kernel is loaded).
void* lookup(const std::string& src, const char* name, bool block, bool load, int threads, size_t smem, int* occ);

// Queue the compilation of `src` as relocatable device code (NVRTC -rdc,
// defining the extern "C" __device__ function `name`); returns its cache key
// ("" when NVRTC is unavailable or the compiler is shut down).
std::string queue_device_fn(const std::string& src, const char* name);

// The cubin link_module would load (no device needed): `base` linked with the
// dispatcher (compiled here) and the compiled functions `keys`; empty on
// failure (last_log says why; *pending, if given, is set when the failure is
// only that some functions are still compiling).  block: wait for the
// functions' compilations.
std::string link_cubin(const void* base, size_t base_size, const std::string& dispatcher,
                       const std::vector<std::string>& keys, bool block, bool* pending = nullptr);

// Link the relocatable cubin `base` (the batch kernel), the `dispatcher`
// source (compiled here) and the queued device functions `keys` with
// nvJitLink into one module, load it on the current device and return its
// kernel `kernel` (cached under link_key per device); *occ <- resident blocks
// per SM at `threads` threads and `smem` dynamic shared memory.  block: wait
// for the queued compilations; load == false (stream capture): only an
// already linked kernel is returned.  Null on failure (last_log says why);
// after a failure other than pending compilations it stays null for link_key.
void* link_module(uint64_t link_key, const void* base, size_t base_size, const std::string& dispatcher,
                  const std::vector<std::string>& keys, const char* kernel, bool block, bool load, int threads,
                  size_t smem, int* occ);

// cuLaunchKernel of a looked-up function; `params` points to the kernel's
// parameter values (one pointer per kernel argument).
int launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t st, void** params);

// Wait for every queued compilation (seconds; < 0: no limit).  QS_ETIMEOUT
// when the limit passed first.
int wait_all(double timeout_s);

// Counters: [0] kernels compiled, [1] compilations failed, [2] queued or
// running, [3] launches of compiled kernels, [4] launches that fell back to
// the generic kernel while a compilation was pending, [5] total compile
// milliseconds, [6] cache hits on a compiled kernel.
void stats(int64_t* out, int n);
// Drop queued compilations and wait for running ones; later lookups of new
// sources stay uncompiled (the generic kernels run them).
void shutdown();
void count_launch(bool compiled);
const char* last_log();

}  // namespace jit
}  // namespace qs
