// up_jit.cpp — NVRTC compile to CUBIN for sm_100a, module cache, loading.
//
// Replaces the reference's AriesDynamicKernelManager (DynamicKernel.h:50-117,
// DynamicKernel.cu:10-158): there, NVRTC produced PTX for compute_XY, which
// was linked with libariesdatatype.a and loaded on every device, with an LRU
// of 100 modules keyed by the full source.  Here NVRTC emits a CUBIN for
// sm_100a directly (the device arithmetic is a header compiled into each
// kernel, so there is no link step), the cubin is cached in memory (LRU keyed
// by the source) and on disk, and it is loaded once with the runtime's
// context-independent cudaLibraryLoadData, whose kernel handles are valid on
// every device of the process.
#include <cuda_runtime.h>
#include <nvJitLink.h>
#include <nvrtc.h>
#include <dlfcn.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <atomic>
#include <list>
#include <map>
#include <mutex>
#include <sstream>
#include <thread>
#include <unordered_map>

#include <zlib.h>

#include "up_internal.h"

namespace upi {

#include "up_dev_embed.inc"  // defines kUpDevCuh and kUpKargsH (the texts of up_dev.cuh and up_kargs.h)

const std::string& device_header_source() {
    static const std::string s(kUpDevCuh);
    return s;
}

const std::string& kargs_header_source() {
    static const std::string s(kUpKargsH);
    return s;
}

struct JitKernelSet {
    std::vector<char> cubin;
    cudaLibrary_t lib = nullptr;
    std::map<std::string, cudaKernel_t> kernels;
    ~JitKernelSet() {
        if (lib) cudaLibraryUnload(lib);
    }
};

namespace {

uint64_t fnv1a(const std::string& s) {
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : s) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h;
}

const char* kArch = "--gpu-architecture=sm_100a";

// Default: <package>/_jitcache beside <package>/_lib/libultraprecise.so, so
// cubins compiled at build time travel with the library; UP_JIT_CACHE_DIR
// overrides it.
std::string cache_dir() {
    const char* d = getenv("UP_JIT_CACHE_DIR");
    if (d && *d) return d;
    Dl_info info;
    if (dladdr((void*)&cache_dir, &info) && info.dli_fname) {
        std::string p = info.dli_fname;
        size_t k = p.rfind('/');
        if (k != std::string::npos) {
            std::string libdir = p.substr(0, k);
            size_t k2 = libdir.rfind('/');
            if (k2 != std::string::npos) return libdir.substr(0, k2) + "/_jitcache";
        }
    }
    const char* home = getenv("HOME");
    return std::string(home && *home ? home : "/tmp") + "/.cache/ultraprecise_b200";
}

bool disk_cache_enabled() {
    const char* e = getenv("UP_JIT_DISK_CACHE");
    return !(e && e[0] == '0');
}

void mkdirs(const std::string& path) {
    std::string cur;
    std::stringstream ss(path);
    std::string part;
    if (!path.empty() && path[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
}

// The cache key covers everything that decides the CUBIN: target, options,
// the NVRTC version, the device library header the source includes, and the
// source itself.
std::string full_key(const std::string& src, bool rdc) {
    int maj = 0, min = 0;
    nvrtcVersion(&maj, &min);
    static const std::string hdr_hash = [] {
        char b[40];
        snprintf(b, sizeof b, "%016llx", (unsigned long long)fnv1a(device_header_source() + kargs_header_source()));
        return std::string(b);
    }();
    return std::string(kArch) + (rdc ? "|rdc" : "") + "|nvrtc" + std::to_string(maj) + "." + std::to_string(min) +
           "|hdr" + hdr_hash + "|" + src;
}

bool read_file_plain(const std::string& p, std::string& out) {
    std::ifstream f(p, std::ios::binary);
    if (!f) return false;
    std::ostringstream o;
    o << f.rdbuf();
    out = o.str();
    return true;
}

// A cache file, or its gzip-compressed form `p.gz` (the in-tree cache that
// travels with the library is stored compressed).
bool read_file(const std::string& p, std::string& out) {
    if (read_file_plain(p, out)) return true;
    gzFile z = gzopen((p + ".gz").c_str(), "rb");
    if (!z) return false;
    out.clear();
    char buf[1 << 16];
    int n;
    while ((n = gzread(z, buf, sizeof buf)) > 0) out.append(buf, (size_t)n);
    const bool ok = n == 0;
    gzclose(z);
    return ok;
}

void write_file_atomic(const std::string& p, const std::string& data) {
    std::string tmp = p + ".tmp." + std::to_string(getpid());
    {
        std::ofstream f(tmp, std::ios::binary);
        if (!f) return;
        f.write(data.data(), (std::streamsize)data.size());
    }
    rename(tmp.c_str(), p.c_str());
}

// Look up entry `name` (a .key file holding the full key beside a .cubin)
// in the cache directory; on a miss, in UP_JIT_CACHE_SEED_DIR, copying a hit
// into the cache directory (used to rebuild a cache with only the entries a
// set of compiles still uses).
bool cache_lookup(const std::string& name, const std::string& key, std::string& bin) {
    const std::string base = cache_dir() + "/" + name;
    std::string k2;
    if (read_file(base + ".key", k2) && k2 == key && read_file(base + ".cubin", bin) && !bin.empty()) return true;
    const char* seed = getenv("UP_JIT_CACHE_SEED_DIR");
    if (!seed || !*seed) return false;
    const std::string sb = std::string(seed) + "/" + name;
    if (read_file(sb + ".key", k2) && k2 == key && read_file(sb + ".cubin", bin) && !bin.empty()) {
        mkdirs(cache_dir());
        write_file_atomic(base + ".cubin", bin);
        write_file_atomic(base + ".key", key);
        return true;
    }
    return false;
}

up_status nvrtc_compile(const std::string& src, std::vector<char>& cubin, std::string& log, bool rdc) {
    nvrtcProgram prog;
    const char* hdr_src[2] = {device_header_source().c_str(), kargs_header_source().c_str()};
    const char* hdr_name[2] = {"up_dev.cuh", "up_kargs.h"};
    nvrtcResult r = nvrtcCreateProgram(&prog, src.c_str(), "up_kernel.cu", 2, hdr_src, hdr_name);
    if (r != NVRTC_SUCCESS) return fail(UP_ERR_COMPILE, std::string("nvrtcCreateProgram: ") + nvrtcGetErrorString(r));
    // UP_JIT_VERBOSE=1 adds ptxas's resource report (registers, spills,
    // shared memory per kernel) and prints the compile log to stderr.
    const char* vb = getenv("UP_JIT_VERBOSE");
    const bool verbose = vb && *vb && *vb != '0';
    // UP_JIT_DUMP_SOURCE=<file> appends every generated kernel source compiled
    if (const char* dump = getenv("UP_JIT_DUMP_SOURCE")) {
        if (FILE* f = fopen(dump, "a")) {
            fprintf(f, "// ---- generated module ----\n%s\n", src.c_str());
            fclose(f);
        }
    }
    std::vector<const char*> opts = {kArch, "-std=c++17", "-lineinfo", "--restrict", "-DUP_NVRTC=1"};
    if (rdc) opts.push_back("-rdc=true");
    if (verbose) opts.push_back("--ptxas-options=-v");
    r = nvrtcCompileProgram(prog, (int)opts.size(), opts.data());
    size_t ls = 0;
    nvrtcGetProgramLogSize(prog, &ls);
    log.assign(ls, '\0');
    if (ls) nvrtcGetProgramLog(prog, &log[0]);
    if (verbose) fprintf(stderr, "%s\n", log.c_str());
    if (r != NVRTC_SUCCESS) {
        nvrtcDestroyProgram(&prog);
        return fail(UP_ERR_COMPILE, "NVRTC: " + std::string(nvrtcGetErrorString(r)) + "\n" + log);
    }
    size_t n = 0;
    r = nvrtcGetCUBINSize(prog, &n);
    if (r != NVRTC_SUCCESS || n == 0) {
        nvrtcDestroyProgram(&prog);
        return fail(UP_ERR_COMPILE, "NVRTC produced no CUBIN");
    }
    cubin.resize(n);
    nvrtcGetCUBIN(prog, cubin.data());
    nvrtcDestroyProgram(&prog);
    return UP_OK;
}

struct Cache {
    std::mutex mu;
    std::list<std::string> lru;  // most recent at front
    std::unordered_map<std::string, std::pair<std::shared_ptr<JitKernelSet>, std::list<std::string>::iterator>> map;
    size_t cap = 256;
};

Cache& cache() {
    static Cache* c = new Cache();  // intentionally leaked: outlives static destructors
    return *c;
}

}  // namespace

// Compile (or read from the disk cache) one source to a CUBIN; with rdc the
// CUBIN is relocatable, for linking with others by nvJitLink.
up_status jit_compile_unit(const std::string& src, bool rdc, std::vector<char>& cubin) {
    const std::string key = full_key(src, rdc);
    const uint64_t h = fnv1a(key);
    char name[32];
    snprintf(name, sizeof name, "%016llx", (unsigned long long)h);
    std::string dir = cache_dir();
    std::string base = dir + "/" + name;
    const char* vb = getenv("UP_JIT_VERBOSE");
    if (disk_cache_enabled() && !(vb && *vb && *vb != '0')) {
        std::string bin;
        if (cache_lookup(name, key, bin)) {
            cubin.assign(bin.begin(), bin.end());
            return UP_OK;
        }
    }
    std::string log;
    up_status st = nvrtc_compile(src, cubin, log, rdc);
    if (st != UP_OK) return st;
    if (disk_cache_enabled()) {
        mkdirs(dir);
        write_file_atomic(base + ".cubin", std::string(cubin.begin(), cubin.end()));
        write_file_atomic(base + ".key", key);
    }
    return UP_OK;
}

up_status jit_compile_cubin(const std::string& src, std::vector<char>& cubin) {
    return jit_compile_unit(src, false, cubin);
}

// nvJitLink is resolved at run time from the CUDA toolkit by absolute path
// (another copy with the same soname may already be loaded by a framework),
// under the versioned names its header maps the API to.
#define UP_STR2(x) #x
#define UP_STR(x) UP_STR2(x)
struct JitLinkApi {
    decltype(&nvJitLinkCreate) create = nullptr;
    decltype(&nvJitLinkAddData) add = nullptr;
    decltype(&nvJitLinkComplete) complete = nullptr;
    decltype(&nvJitLinkGetLinkedCubinSize) cubin_size = nullptr;
    decltype(&nvJitLinkGetLinkedCubin) cubin = nullptr;
    decltype(&nvJitLinkGetErrorLogSize) log_size = nullptr;
    decltype(&nvJitLinkGetErrorLog) log = nullptr;
    decltype(&nvJitLinkDestroy) destroy = nullptr;
    decltype(&nvJitLinkGetInfoLogSize) info_size = nullptr;
    decltype(&nvJitLinkGetInfoLog) info = nullptr;
    bool ok = false;
};

const JitLinkApi& jitlink() {
    static JitLinkApi api = [] {
        JitLinkApi a;
        std::vector<std::string> paths;
        if (const char* ch = getenv("CUDA_HOME")) paths.push_back(std::string(ch) + "/lib64/libnvJitLink.so.12");
        paths.push_back("/usr/local/cuda/lib64/libnvJitLink.so.12");
        paths.push_back("libnvJitLink.so.12");
        void* h = nullptr;
        for (const auto& p : paths)
            if ((h = dlopen(p.c_str(), RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) return a;
        a.create = (decltype(a.create))dlsym(h, UP_STR(nvJitLinkCreate));
        a.add = (decltype(a.add))dlsym(h, UP_STR(nvJitLinkAddData));
        a.complete = (decltype(a.complete))dlsym(h, UP_STR(nvJitLinkComplete));
        a.cubin_size = (decltype(a.cubin_size))dlsym(h, UP_STR(nvJitLinkGetLinkedCubinSize));
        a.cubin = (decltype(a.cubin))dlsym(h, UP_STR(nvJitLinkGetLinkedCubin));
        a.log_size = (decltype(a.log_size))dlsym(h, UP_STR(nvJitLinkGetErrorLogSize));
        a.log = (decltype(a.log))dlsym(h, UP_STR(nvJitLinkGetErrorLog));
        a.destroy = (decltype(a.destroy))dlsym(h, UP_STR(nvJitLinkDestroy));
        a.info_size = (decltype(a.info_size))dlsym(h, UP_STR(nvJitLinkGetInfoLogSize));
        a.info = (decltype(a.info))dlsym(h, UP_STR(nvJitLinkGetInfoLog));
        a.ok = a.create && a.add && a.complete && a.cubin_size && a.cubin && a.log_size && a.log && a.destroy;
        return a;
    }();
    return api;
}

// Compile every unit (relocatable, cached per unit, in parallel) and link
// them with nvJitLink; the linked CUBIN is cached under the units' keys.
up_status jit_compile_linked(const std::vector<std::string>& units, std::vector<char>& linked) {
    std::string all;
    for (const auto& u : units) all += full_key(u, true) + "\x1f";
    const std::string key = "linked|" + all;
    char name[40];
    snprintf(name, sizeof name, "L%016llx", (unsigned long long)fnv1a(key));
    const std::string base = cache_dir() + "/" + name;
    // UP_JIT_LINK_VERBOSE=1 relinks and prints the linker's per-kernel
    // resource report (registers, stack frame, whether the call graph's stack
    // size could be determined) to stderr.
    const char* vb = getenv("UP_JIT_LINK_VERBOSE");
    const bool verbose = vb && *vb && *vb != '0';
    if (disk_cache_enabled() && !verbose) {
        std::string bin;
        if (cache_lookup(name, key, bin)) {
            linked.assign(bin.begin(), bin.end());
            return UP_OK;
        }
    }
    std::vector<std::vector<char>> objs(units.size());
    std::vector<up_status> sts(units.size(), UP_OK);
    std::vector<std::string> errs(units.size());
    {
        unsigned nthr = std::max(1u, std::min<unsigned>(std::thread::hardware_concurrency(), 32u));
        std::vector<std::thread> pool;
        std::atomic<size_t> next{0};
        for (unsigned t = 0; t < nthr; t++)
            pool.emplace_back([&]() {
                for (size_t i; (i = next.fetch_add(1)) < units.size();) {
                    sts[i] = jit_compile_unit(units[i], true, objs[i]);
                    if (sts[i] != UP_OK) errs[i] = last_error();
                }
            });
        for (auto& th : pool) th.join();
    }
    for (size_t i = 0; i < units.size(); i++)
        if (sts[i] != UP_OK) return fail(sts[i], "unit " + std::to_string(i) + ": " + errs[i]);
    const JitLinkApi& L = jitlink();
    if (!L.ok) return fail(UP_ERR_COMPILE, "libnvJitLink.so.12 not found (needed to link batch modules)");
    nvJitLinkHandle h;
    const char* lopts[] = {"-arch=sm_100a", "-verbose"};
    if (L.create(&h, verbose ? 2 : 1, lopts) != NVJITLINK_SUCCESS) return fail(UP_ERR_COMPILE, "nvJitLinkCreate failed");
    nvJitLinkResult lr = NVJITLINK_SUCCESS;
    for (size_t i = 0; i < objs.size() && lr == NVJITLINK_SUCCESS; i++)
        lr = L.add(h, NVJITLINK_INPUT_CUBIN, objs[i].data(), objs[i].size(), ("unit" + std::to_string(i)).c_str());
    if (lr == NVJITLINK_SUCCESS) lr = L.complete(h);
    if (lr != NVJITLINK_SUCCESS) {
        size_t ls = 0;
        L.log_size(h, &ls);
        std::string log(ls, '\0');
        if (ls) L.log(h, &log[0]);
        L.destroy(&h);
        return fail(UP_ERR_COMPILE, "nvJitLink: " + log);
    }
    if (verbose && L.info_size && L.info) {
        size_t is = 0;
        L.info_size(h, &is);
        std::string info(is, '\0');
        if (is) L.info(h, &info[0]);
        fprintf(stderr, "%s\n", info.c_str());
    }
    size_t n = 0;
    L.cubin_size(h, &n);
    linked.resize(n);
    L.cubin(h, linked.data());
    L.destroy(&h);
    if (disk_cache_enabled()) {
        mkdirs(cache_dir());
        write_file_atomic(base + ".cubin", std::string(linked.begin(), linked.end()));
        write_file_atomic(base + ".key", key);
    }
    return UP_OK;
}

// Kernels that keep wide limb arrays in a stack frame may need more than the
// context's default per-thread stack (1 KB); when they do, a launch makes the
// driver grow local memory.  Raise the context's limit once, at load time, to
// the largest frame of the module's kernels.
void fit_stack_limit(const JitKernelSet& ks) {
    static std::mutex mu;
    size_t need = 0;
    for (const auto& kv : ks.kernels) {
        cudaFuncAttributes fa;
        if (cudaFuncGetAttributes(&fa, (const void*)kv.second) == cudaSuccess) need = std::max(need, fa.localSizeBytes);
        else cudaGetLastError();
    }
    std::lock_guard<std::mutex> g(mu);
    size_t have = 0;
    if (cudaDeviceGetLimit(&have, cudaLimitStackSize) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    if (need > have && cudaDeviceSetLimit(cudaLimitStackSize, (need + 255) & ~(size_t)255) != cudaSuccess)
        cudaGetLastError();
}

// Load an already compiled CUBIN and look up its kernels.
up_status jit_load(const std::vector<char>& cubin, const std::vector<std::string>& kernels,
                   std::shared_ptr<JitKernelSet>& out) {
    auto ks = std::make_shared<JitKernelSet>();
    ks->cubin = cubin;
    cudaError_t e = cudaLibraryLoadData(&ks->lib, ks->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) {
        ks->lib = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                    std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e));
    }
    for (const auto& k : kernels) {
        cudaKernel_t h = nullptr;
        e = cudaLibraryGetKernel(&h, ks->lib, k.c_str());
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(UP_ERR_CUDA, "cudaLibraryGetKernel(" + k + "): " + cudaGetErrorString(e));
        }
        ks->kernels[k] = h;
    }
    fit_stack_limit(*ks);
    out = ks;
    return UP_OK;
}

up_status jit_get(const GeneratedModule& gen, std::shared_ptr<JitKernelSet>& out) {
    Cache& c = cache();
    {
        std::lock_guard<std::mutex> g(c.mu);
        auto it = c.map.find(gen.source);
        if (it != c.map.end()) {
            c.lru.erase(it->second.second);
            c.lru.push_front(gen.source);
            it->second.second = c.lru.begin();
            out = it->second.first;
            return UP_OK;
        }
    }
    auto ks = std::make_shared<JitKernelSet>();
    up_status st = jit_compile_cubin(gen.source, ks->cubin);
    if (st != UP_OK) return st;
    cudaError_t e = cudaLibraryLoadData(&ks->lib, ks->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
    if (e != cudaSuccess) {
        ks->lib = nullptr;
        cudaGetLastError();
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? UP_ERR_NO_DEVICE : UP_ERR_CUDA,
                    std::string("cudaLibraryLoadData: ") + cudaGetErrorString(e));
    }
    for (const auto& k : gen.kernels) {
        cudaKernel_t h = nullptr;
        e = cudaLibraryGetKernel(&h, ks->lib, k.c_str());
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(UP_ERR_CUDA, "cudaLibraryGetKernel(" + k + "): " + cudaGetErrorString(e));
        }
        ks->kernels[k] = h;
    }
    fit_stack_limit(*ks);
    std::lock_guard<std::mutex> g(c.mu);
    auto it = c.map.find(gen.source);
    if (it != c.map.end()) {  // another thread won the race
        out = it->second.first;
        return UP_OK;
    }
    c.lru.push_front(gen.source);
    c.map[gen.source] = {ks, c.lru.begin()};
    while (c.map.size() > c.cap) {
        c.map.erase(c.lru.back());
        c.lru.pop_back();
    }
    out = ks;
    return UP_OK;
}

void* jit_kernel(const JitKernelSet& ks, const std::string& name) {
    auto it = ks.kernels.find(name);
    return it == ks.kernels.end() ? nullptr : (void*)it->second;
}

int jit_cache_size(bool clear) {
    Cache& c = cache();
    std::lock_guard<std::mutex> g(c.mu);
    int n = (int)c.map.size();
    if (clear) {
        c.map.clear();
        c.lru.clear();
    }
    return n;
}

}  // namespace upi
