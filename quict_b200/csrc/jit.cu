// Run-time compilation of generated pass kernels (see jit.h).
//
// A source string is compiled once per process by NVRTC into an sm_100a cubin
// (on a small pool of host threads), and the cubin is loaded once per device
// with cuModuleLoadData.  Sources are keyed by their full text, so two passes
// with the same structure share one kernel whatever their matrices are (the
// matrices travel in the launch's parameter block).
#include <dlfcn.h>

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include <cuda.h>
#include <nvJitLink.h>
#include <nvrtc.h>

#include "common.cuh"
#include "jit.h"

namespace qs {
namespace jit {
namespace {

struct Api {
    bool nvrtc_tried = false, nvrtc_ok = false, cu_tried = false, cu_ok = false;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    decltype(&nvrtcGetErrorString) nvrtc_err = nullptr;
    decltype(&cuModuleLoadData) module_load = nullptr;
    decltype(&cuModuleGetFunction) get_function = nullptr;
    decltype(&cuLaunchKernel) launch_kernel = nullptr;
    decltype(&cuFuncSetAttribute) set_attr = nullptr;
    decltype(&cuOccupancyMaxActiveBlocksPerMultiprocessor) occupancy = nullptr;
    decltype(&cuGetErrorString) cu_err = nullptr;
};

void* open_first(const char* const* names) {
    for (int i = 0; names[i]; ++i)
        if (void* h = dlopen(names[i], RTLD_NOW | RTLD_LOCAL)) return h;
    return nullptr;
}

template <typename F>
bool sym(void* h, const char* name, F& out) {
    out = reinterpret_cast<F>(dlsym(h, name));
    return out != nullptr;
}

struct Entry {
    std::string src, name;
    bool rdc = false;  // relocatable device code (a __device__ function for the linked batch kernel)
    int state = 0;  // 0 queued or compiling, 1 ready, 2 failed
    std::string cubin, log;
    double ms = 0.0;
    void* mod[64] = {nullptr};
    void* fn[64] = {nullptr};
    int occ[64] = {0};
};

// nvJitLink, opened with dlopen like NVRTC (the versioned names its header
// maps the API to).
struct LinkApi {
    bool tried = false, ok = false;
    decltype(&__nvJitLinkCreate_12_9) create = nullptr;
    decltype(&__nvJitLinkAddData_12_9) add = nullptr;
    decltype(&__nvJitLinkComplete_12_9) complete = nullptr;
    decltype(&__nvJitLinkGetLinkedCubinSize_12_9) cubin_size = nullptr;
    decltype(&__nvJitLinkGetLinkedCubin_12_9) cubin = nullptr;
    decltype(&__nvJitLinkGetErrorLogSize_12_9) log_size = nullptr;
    decltype(&__nvJitLinkGetErrorLog_12_9) log = nullptr;
    decltype(&__nvJitLinkDestroy_12_9) destroy = nullptr;
};

// A linked module (the batch kernel with its device functions) per device.
struct Linked {
    void* mod[64] = {nullptr};
    void* fn[64] = {nullptr};
    int occ[64] = {0};
    bool failed = false;  // a link or load failed once: callers run the generic kernel from then on
};

struct State {
    std::mutex mu;  // guards everything below and the API tables
    std::condition_variable cv;
    Api api;
    LinkApi link;
    std::unordered_map<uint64_t, std::shared_ptr<Linked>> linked;
    // keyed by a 128-bit hash of the source text (the text itself is kept
    // only until the entry is compiled)
    std::unordered_map<std::string, std::shared_ptr<Entry>> cache;
    std::deque<std::shared_ptr<Entry>> queue;
    int workers = 0;
    int pending = 0;
    int running = 0;
    bool stopping = false;
    std::string last_log;
    std::atomic<int> mode{-1};
    std::atomic<int64_t> compiled{0}, failed{0}, jit_launches{0}, fallback_launches{0}, hits{0};
    std::atomic<int64_t> compile_us{0};
};

// 128-bit key of a source text: two independent 64-bit FNV-1a hashes.
std::string source_key(const std::string& src) {
    uint64_t a = 1469598103934665603ull, b = 0x9e3779b97f4a7c15ull;
    for (unsigned char c : src) {
        a = (a ^ c) * 1099511628211ull;
        b = (b ^ c) * 0x100000001b3ull + 0x632be59bd9b4e019ull;
    }
    return std::string(reinterpret_cast<const char*>(&a), 8) + std::string(reinterpret_cast<const char*>(&b), 8) +
           std::to_string(src.size());
}

// Never destroyed: worker threads may still run while the process exits.
State& S() {
    static State* s = new State();
    return *s;
}

bool load_nvrtc(State& s) {  // with s.mu held
    if (s.api.nvrtc_tried) return s.api.nvrtc_ok;
    s.api.nvrtc_tried = true;
    static const char* names[] = {"libnvrtc.so.12", "libnvrtc.so", nullptr};
    void* h = open_first(names);
    Api& a = s.api;
    a.nvrtc_ok = h && sym(h, "nvrtcCreateProgram", a.create) && sym(h, "nvrtcCompileProgram", a.compile) &&
                 sym(h, "nvrtcGetCUBINSize", a.cubin_size) && sym(h, "nvrtcGetCUBIN", a.cubin) &&
                 sym(h, "nvrtcGetProgramLogSize", a.log_size) && sym(h, "nvrtcGetProgramLog", a.log) &&
                 sym(h, "nvrtcDestroyProgram", a.destroy) && sym(h, "nvrtcGetErrorString", a.nvrtc_err);
    if (!a.nvrtc_ok) s.last_log = "NVRTC (libnvrtc.so.12) is not available";
    return a.nvrtc_ok;
}

bool load_driver(State& s) {  // with s.mu held
    if (s.api.cu_tried) return s.api.cu_ok;
    s.api.cu_tried = true;
    static const char* names[] = {"libcuda.so.1", "libcuda.so", nullptr};
    void* h = open_first(names);
    Api& a = s.api;
    a.cu_ok = h && sym(h, "cuModuleLoadData", a.module_load) && sym(h, "cuModuleGetFunction", a.get_function) &&
              sym(h, "cuLaunchKernel", a.launch_kernel) && sym(h, "cuFuncSetAttribute", a.set_attr) &&
              sym(h, "cuOccupancyMaxActiveBlocksPerMultiprocessor", a.occupancy) &&
              sym(h, "cuGetErrorString", a.cu_err);
    if (!a.cu_ok) s.last_log = "the CUDA driver library (libcuda.so.1) is not available";
    return a.cu_ok;
}

// The newest versioned name (__<base>_12_9 .. _12_0) the library exports.
template <typename F>
bool sym_versioned(void* h, const char* base, F& out) {
    for (int minor = 9; minor >= 0; --minor) {
        char nm[96];
        snprintf(nm, sizeof(nm), "__%s_12_%d", base, minor);
        if (sym(h, nm, out)) return true;
    }
    return false;
}

bool load_link(State& s) {  // with s.mu held
    if (s.link.tried) return s.link.ok;
    s.link.tried = true;
    // The toolkit's copy first, by path: a framework imported earlier may have
    // loaded an older libnvJitLink.so.12 under the same name.
    std::string tk = std::string(getenv("CUDA_HOME") && *getenv("CUDA_HOME") ? getenv("CUDA_HOME") : "/usr/local/cuda") +
                     "/lib64/libnvJitLink.so.12";
    const char* names[] = {tk.c_str(), "libnvJitLink.so.12", "libnvJitLink.so", nullptr};
    void* h = open_first(names);
    LinkApi& a = s.link;
    a.ok = h && sym_versioned(h, "nvJitLinkCreate", a.create) && sym_versioned(h, "nvJitLinkAddData", a.add) &&
           sym_versioned(h, "nvJitLinkComplete", a.complete) &&
           sym_versioned(h, "nvJitLinkGetLinkedCubinSize", a.cubin_size) &&
           sym_versioned(h, "nvJitLinkGetLinkedCubin", a.cubin) &&
           sym_versioned(h, "nvJitLinkGetErrorLogSize", a.log_size) &&
           sym_versioned(h, "nvJitLinkGetErrorLog", a.log) && sym_versioned(h, "nvJitLinkDestroy", a.destroy);
    if (!a.ok) s.last_log = "nvJitLink (libnvJitLink.so.12) is not available";
    return a.ok;
}

// Compile `e` (no lock held while NVRTC runs).
void compile_entry(State& s, Entry& e) {
    auto t0 = std::chrono::steady_clock::now();
    Api& a = s.api;
    nvrtcProgram prog = nullptr;
    std::string log, cubin;
    bool ok = a.create(&prog, e.src.c_str(), "qs_pass.cu", 0, nullptr, nullptr) == NVRTC_SUCCESS;
    if (ok) {
        // QS_JIT_OPTS: extra NVRTC options, space separated (e.g. --ptxas-options=-v)
        std::vector<std::string> extra;
        if (const char* env = getenv("QS_JIT_OPTS")) {
            std::string cur;
            for (const char* c = env;; ++c) {
                if (*c == ' ' || *c == 0) {
                    if (!cur.empty()) extra.push_back(cur);
                    cur.clear();
                    if (*c == 0) break;
                } else {
                    cur += *c;
                }
            }
        }
        std::vector<const char*> opts = {"-arch=sm_100a", "-std=c++17", "-w"};
        if (e.rdc) opts.push_back("-rdc=true");
        for (const auto& x : extra) opts.push_back(x.c_str());
        nvrtcResult r = a.compile(prog, int(opts.size()), opts.data());
        size_t ls = 0;
        if (a.log_size(prog, &ls) == NVRTC_SUCCESS && ls > 1) {
            log.resize(ls);
            a.log(prog, &log[0]);
        }
        ok = r == NVRTC_SUCCESS;
        if (!ok) log = std::string(a.nvrtc_err(r)) + "\n" + log;
        size_t cs = 0;
        if (ok && a.cubin_size(prog, &cs) == NVRTC_SUCCESS && cs > 0) {
            cubin.resize(cs);
            ok = a.cubin(prog, &cubin[0]) == NVRTC_SUCCESS;
        } else {
            ok = false;
        }
        a.destroy(&prog);
    } else {
        log = "nvrtcCreateProgram failed";
    }
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::lock_guard<std::mutex> lock(s.mu);
    e.ms = ms;
    e.log = log;
    s.compile_us += int64_t(ms * 1e3);
    if (ok) {
        e.cubin.swap(cubin);
        e.state = 1;
        ++s.compiled;
        std::string().swap(e.src);  // the cache keeps the hash, not the text
    } else {
        e.state = 2;
        ++s.failed;
        s.last_log = "compile of " + e.name + " failed: " + log.substr(0, 4000);
    }
    --s.pending;
    s.cv.notify_all();
}

void worker_loop() {
    State& s = S();
    for (;;) {
        std::shared_ptr<Entry> e;
        {
            // after shutdown_workers the thread parks here until the process
            // ends: a returning thread would run the compiler library's
            // thread-exit hooks while the process is unloading that library
            std::unique_lock<std::mutex> lock(s.mu);
            s.cv.wait(lock, [&] { return !s.queue.empty() && !s.stopping; });
            e = s.queue.front();
            s.queue.pop_front();
            ++s.running;
        }
        compile_entry(s, *e);
        std::lock_guard<std::mutex> lock(s.mu);
        --s.running;
        s.cv.notify_all();
    }
}

// At process exit: drop queued work and let running compilations finish, so
// no worker is inside NVRTC while the process tears its libraries down (the
// idle workers stay parked; the process ends them).
void shutdown_workers() {
    State& s = S();
    std::unique_lock<std::mutex> lock(s.mu);
    if (s.stopping && s.running == 0) return;
    s.stopping = true;
    for (auto& e : s.queue) e->state = 2;
    s.pending -= int(s.queue.size());
    s.queue.clear();
    s.cv.notify_all();
    s.cv.wait_for(lock, std::chrono::seconds(120), [&] { return s.running == 0; });
}

void start_workers(State& s) {  // with s.mu held
    if (s.workers > 0) return;
    unsigned hw = std::thread::hardware_concurrency();
    int n = hw > 2 ? int(hw) - 1 : 1;
    if (n > 16) n = 16;
    for (int i = 0; i < n; ++i) std::thread(worker_loop).detach();
    s.workers = n;
    std::atexit(shutdown_workers);
}

// Loaded function of a ready entry on the current device (with s.mu held);
// loads it when `load` allows.
void* device_function(State& s, Entry& e, bool load, int threads, size_t smem, int* occ) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    if (e.fn[dev]) {
        *occ = e.occ[dev];
        return e.fn[dev];
    }
    if (!load || !load_driver(s)) return nullptr;
    cudaFree(nullptr);  // the runtime's primary context is current from here on
    CUmodule mod = nullptr;
    CUresult r = s.api.module_load(&mod, e.cubin.data());
    if (r != CUDA_SUCCESS) {
        const char* m = nullptr;
        s.api.cu_err(r, &m);
        s.last_log = std::string("cuModuleLoadData: ") + (m ? m : "error");
        e.state = 2;
        return nullptr;
    }
    CUfunction fn = nullptr;
    r = s.api.get_function(&fn, mod, e.name.c_str());
    if (r != CUDA_SUCCESS) {
        s.last_log = "cuModuleGetFunction failed for " + e.name;
        e.state = 2;
        return nullptr;
    }
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (optin > 0) s.api.set_attr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, optin);
    int nb = 0;
    if (s.api.occupancy(&nb, fn, threads, smem) != CUDA_SUCCESS || nb < 1) {
        s.last_log = "cuOccupancyMaxActiveBlocksPerMultiprocessor: the kernel does not fit an SM";
        e.state = 2;
        return nullptr;
    }
    e.mod[dev] = mod;
    e.fn[dev] = fn;
    e.occ[dev] = nb;
    *occ = nb;
    return fn;
}

}  // namespace

int mode() {
    State& s = S();
    int m = s.mode.load();
    if (m < 0) {
        const char* env = getenv("QS_JIT");
        m = env && *env ? atoi(env) : QS_JIT_ASYNC;
        if (m < QS_JIT_OFF || m > QS_JIT_SYNC) m = QS_JIT_ASYNC;
        s.mode = m;
    }
    return m;
}

void set_mode(int m) { S().mode = m; }

void shutdown() {
    State& s = S();
    {
        std::lock_guard<std::mutex> lock(s.mu);
        if (s.workers == 0) return;
    }
    shutdown_workers();
}

void* lookup(const std::string& src, const char* name, bool block, bool load, int threads, size_t smem, int* occ) {
    State& s = S();
    std::shared_ptr<Entry> e;
    bool compile_here = false;
    {
        std::unique_lock<std::mutex> lock(s.mu);
        if (!load_nvrtc(s)) return nullptr;
        const std::string key = source_key(src);
        if (s.stopping && s.cache.find(key) == s.cache.end()) return nullptr;  // shut down: nothing new
        auto it = s.cache.find(key);
        if (it == s.cache.end()) {
            e = std::make_shared<Entry>();
            e->src = src;
            e->name = name;
            s.cache.emplace(key, e);
            ++s.pending;
            if (block) {
                compile_here = true;
            } else {
                start_workers(s);
                s.queue.push_back(e);
                s.cv.notify_all();
                return nullptr;
            }
        } else {
            e = it->second;
        }
        if (!compile_here) {
            if (e->state == 0 && block) s.cv.wait(lock, [&] { return e->state != 0; });
            if (e->state != 1) return nullptr;
            ++s.hits;
            return device_function(s, *e, load, threads, smem, occ);
        }
    }
    compile_entry(s, *e);
    std::lock_guard<std::mutex> lock(s.mu);
    if (e->state != 1) return nullptr;
    return device_function(s, *e, load, threads, smem, occ);
}

std::string queue_device_fn(const std::string& src, const char* name) {
    State& s = S();
    std::unique_lock<std::mutex> lock(s.mu);
    if (!load_nvrtc(s)) return std::string();
    const std::string key = source_key(src) + "r";
    if (s.cache.find(key) != s.cache.end()) return key;
    if (s.stopping) return std::string();
    auto e = std::make_shared<Entry>();
    e->src = src;
    e->name = name;
    e->rdc = true;
    s.cache.emplace(key, e);
    ++s.pending;
    start_workers(s);
    s.queue.push_back(e);
    s.cv.notify_all();
    return key;
}

// The linked cubin of `base`, the dispatcher and the compiled functions
// `keys` (empty on failure, with last_log set).  block: wait for the
// functions' compilations; otherwise fail while any is pending.
std::string link_cubin(const void* base, size_t base_size, const std::string& dispatcher,
                       const std::vector<std::string>& keys, bool block, bool* pending) {
    State& s = S();
    if (pending) *pending = false;
    std::vector<std::shared_ptr<Entry>> es;
    {
        std::unique_lock<std::mutex> lock(s.mu);
        if (!load_nvrtc(s)) return std::string();
        for (const auto& k : keys) {
            auto e = s.cache.find(k);
            if (e == s.cache.end()) {
                s.last_log = "link: a device function was never queued";
                return std::string();
            }
            es.push_back(e->second);
        }
        auto all_done = [&] {
            for (const auto& e : es)
                if (e->state == 0) return false;
            return true;
        };
        if (block) s.cv.wait(lock, all_done);
        if (!all_done()) {
            s.last_log = "link: device functions still compiling";
            if (pending) *pending = true;
            return std::string();
        }
        for (const auto& e : es)
            if (e->state != 1) {
                s.last_log = "link: compile of " + e->name + " failed: " + e->log.substr(0, 3000);
                return std::string();
            }
        if (!load_link(s)) return std::string();
        ++s.pending;  // the dispatcher, compiled below
    }
    Entry d;
    d.src = dispatcher;
    d.name = "qs_batch_dispatch";
    d.rdc = true;
    compile_entry(s, d);
    if (d.state != 1) {
        std::lock_guard<std::mutex> lock(s.mu);
        s.last_log = "link: compile of the dispatcher failed: " + d.log.substr(0, 3000);
        return std::string();
    }
    LinkApi& L = s.link;
    nvJitLinkHandle h = nullptr;
    const char* lopts[] = {"-arch=sm_100a"};
    std::string err;
    bool ok = L.create(&h, 1, lopts) == NVJITLINK_SUCCESS;
    if (ok) ok = L.add(h, NVJITLINK_INPUT_CUBIN, base, base_size, "batch_kernel") == NVJITLINK_SUCCESS;
    if (ok) ok = L.add(h, NVJITLINK_INPUT_CUBIN, d.cubin.data(), d.cubin.size(), "dispatch") == NVJITLINK_SUCCESS;
    for (size_t i = 0; ok && i < es.size(); ++i)  // ready entries' cubins no longer change
        ok = L.add(h, NVJITLINK_INPUT_CUBIN, es[i]->cubin.data(), es[i]->cubin.size(), es[i]->name.c_str()) ==
             NVJITLINK_SUCCESS;
    if (ok) ok = L.complete(h) == NVJITLINK_SUCCESS;
    std::string cubin;
    size_t cs = 0;
    if (ok) ok = L.cubin_size(h, &cs) == NVJITLINK_SUCCESS && cs > 0;
    if (ok) {
        cubin.resize(cs);
        ok = L.cubin(h, &cubin[0]) == NVJITLINK_SUCCESS;
    }
    if (!ok && h) {
        size_t ls = 0;
        if (L.log_size(h, &ls) == NVJITLINK_SUCCESS && ls > 1) {
            err.resize(ls);
            L.log(h, &err[0]);
        }
    }
    if (h) L.destroy(&h);
    if (!ok) {
        std::lock_guard<std::mutex> lock(s.mu);
        s.last_log = "nvJitLink failed: " + err.substr(0, 4000);
        return std::string();
    }
    return cubin;
}

void* link_module(uint64_t link_key, const void* base, size_t base_size, const std::string& dispatcher,
                  const std::vector<std::string>& keys, const char* kernel, bool block, bool load, int threads,
                  size_t smem, int* occ) {
    State& s = S();
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return nullptr;
    std::shared_ptr<Linked> lm;
    {
        std::lock_guard<std::mutex> lock(s.mu);
        auto it = s.linked.find(link_key);
        if (it != s.linked.end() && it->second->fn[dev]) {
            *occ = it->second->occ[dev];
            return it->second->fn[dev];
        }
        if (it != s.linked.end() && it->second->failed) return nullptr;
        if (!load || !load_driver(s)) return nullptr;
        if (it == s.linked.end()) it = s.linked.emplace(link_key, std::make_shared<Linked>()).first;
        lm = it->second;
    }
    bool pending = false;
    const std::string cubin = link_cubin(base, base_size, dispatcher, keys, block, &pending);
    std::lock_guard<std::mutex> lock(s.mu);
    if (cubin.empty()) {
        if (!pending) lm->failed = true;  // still compiling: a later launch tries again; other failures are final
        return nullptr;
    }
    cudaFree(nullptr);  // the runtime's primary context is current from here on
    CUmodule mod = nullptr;
    CUresult r = s.api.module_load(&mod, cubin.data());
    if (r != CUDA_SUCCESS) {
        const char* m = nullptr;
        s.api.cu_err(r, &m);
        s.last_log = std::string("cuModuleLoadData (linked batch kernel): ") + (m ? m : "error");
        lm->failed = true;
        return nullptr;
    }
    CUfunction fn = nullptr;
    if (s.api.get_function(&fn, mod, kernel) != CUDA_SUCCESS) {
        s.last_log = std::string("cuModuleGetFunction failed for ") + kernel;
        lm->failed = true;
        return nullptr;
    }
    int optin = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // the kernel's static shared memory (a few hundred bytes) comes out of the same opt-in limit
    if (optin > 4096) s.api.set_attr(fn, CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES, optin - 4096);
    int nb = 0;
    if (s.api.occupancy(&nb, fn, threads, smem) != CUDA_SUCCESS || nb < 1) {
        s.last_log = "cuOccupancyMaxActiveBlocksPerMultiprocessor: the linked batch kernel does not fit an SM";
        lm->failed = true;
        return nullptr;
    }
    lm->mod[dev] = mod;
    lm->fn[dev] = fn;
    lm->occ[dev] = nb;
    *occ = nb;
    return fn;
}

int launch(void* fn, unsigned grid, unsigned block, size_t smem, cudaStream_t st, void** params) {
    State& s = S();
    CUresult r = s.api.launch_kernel(static_cast<CUfunction>(fn), grid, 1, 1, block, 1, 1, unsigned(smem),
                                     reinterpret_cast<CUstream>(st), params, nullptr);
    if (r != CUDA_SUCCESS) {
        const char* m = nullptr;
        s.api.cu_err(r, &m);
        set_error("cuLaunchKernel (compiled pass): %s", m ? m : "error");
        return QS_ECUDA;
    }
    return QS_OK;
}

int wait_all(double timeout_s) {
    State& s = S();
    std::unique_lock<std::mutex> lock(s.mu);
    auto done = [&] { return s.pending == 0; };
    if (timeout_s < 0) {
        s.cv.wait(lock, done);
        return QS_OK;
    }
    bool ok = s.cv.wait_for(lock, std::chrono::duration<double>(timeout_s), done);
    if (!ok) {
        set_error("qs_jit_wait: %d compilations still pending after %.1f s", s.pending, timeout_s);
        return QS_ETIMEOUT;
    }
    return QS_OK;
}

void stats(int64_t* out, int n) {
    State& s = S();
    int64_t v[7];
    {
        std::lock_guard<std::mutex> lock(s.mu);
        v[2] = s.pending;
    }
    v[0] = s.compiled;
    v[1] = s.failed;
    v[3] = s.jit_launches;
    v[4] = s.fallback_launches;
    v[5] = s.compile_us / 1000;
    v[6] = s.hits;
    for (int i = 0; i < n && i < 7; ++i) out[i] = v[i];
}

void count_launch(bool compiled) {
    if (compiled) ++S().jit_launches;
    else ++S().fallback_launches;
}

const char* last_log() {
    State& s = S();
    std::lock_guard<std::mutex> lock(s.mu);
    static thread_local std::string copy;
    copy = s.last_log;
    return copy.c_str();
}

// NVRTC-only compilation of `src` (no device needed): cubin size or error.
int compile_check(const char* src, int64_t* cubin_bytes, std::string* log) {
    State& s = S();
    {
        std::lock_guard<std::mutex> lock(s.mu);
        if (!load_nvrtc(s)) {
            set_error("qs_jit_compile_check: %s", s.last_log.c_str());
            return QS_ENOTSUP;
        }
    }
    Entry e;
    e.src = src;
    e.name = "check";
    {
        std::lock_guard<std::mutex> lock(s.mu);
        ++s.pending;
    }
    compile_entry(s, e);
    *log = e.log;
    {
        std::lock_guard<std::mutex> lock(s.mu);
        s.last_log = e.log;
    }
    if (e.state != 1) {
        set_error("qs_jit_compile_check: %s", e.log.substr(0, 400).c_str());
        return QS_EINVAL;
    }
    *cubin_bytes = int64_t(e.cubin.size());
    return QS_OK;
}

}  // namespace jit
}  // namespace qs

extern "C" int qs_jit_shutdown(void) {
    qs::jit::shutdown();
    return QS_OK;
}

extern "C" int qs_jit_set_mode(int mode) {
    if (mode < QS_JIT_OFF || mode > QS_JIT_SYNC) {
        qs::set_error("qs_jit_set_mode: mode %d outside [%d, %d]", mode, QS_JIT_OFF, QS_JIT_SYNC);
        return QS_EINVAL;
    }
    const int prev = qs::jit::mode();
    qs::jit::set_mode(mode);
    return prev;
}

extern "C" int qs_jit_wait(double timeout_s) { return qs::jit::wait_all(timeout_s); }

extern "C" int qs_jit_stats(int64_t* out, int n) {
    if (out == nullptr || n < 0) {
        qs::set_error("qs_jit_stats: bad output array");
        return QS_EINVAL;
    }
    qs::jit::stats(out, n);
    return QS_OK;
}

extern "C" const char* qs_jit_last_log(void) { return qs::jit::last_log(); }

extern "C" int qs_jit_compile_check(const char* src, int64_t* cubin_bytes) {
    if (src == nullptr || cubin_bytes == nullptr) {
        qs::set_error("qs_jit_compile_check: null argument");
        return QS_EINVAL;
    }
    std::string log;
    return qs::jit::compile_check(src, cubin_bytes, &log);
}
