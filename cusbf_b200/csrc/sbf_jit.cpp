// sbf_jit.cpp -- kernels for configurations that are not compiled into the
// library.  The reference is header-only, so every Config<K,S,M,H>
// a caller names gets kernels specialised at compile time.  A prebuilt
// library can only hold a few, so for any other configuration the same tile
// kernel source (sbf_tile.cuh and its two headers, embedded in the library
// at build time) is compiled with NVRTC for the device at filter creation,
// loaded with the runtime's library API, and launched like the compiled
// kernels (cudaLaunchKernel accepts a cudaKernel_t).
//
// Compilation takes about ten seconds, so the cubin is cached on disk under
// $SBF_JIT_CACHE (default ~/.cache/sbf_b200), keyed by the configuration, the
// device architecture, the NVRTC version and a hash of the embedded source.
// The protein and DNA-triplet alphabets get the generic kernels
// (sbf_generic.cuh) compiled the same way with the configuration as template
// constants.  SBF_JIT=0 turns this off; then, and on any failure, the filter
// runs the runtime-parameterised generic kernels, which give the same
// results more slowly.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>
#include <sys/stat.h>
#include <unistd.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <set>
#include <sstream>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "../../include/sbf_b200.h"
#include "sbf_host.h"
#include "sbf_internal.h"
#include "sbf_jit_sources.inc"  // kJit* kernel sources (generated)

namespace sbf {
namespace {

// Fixed-width integer types for NVRTC, which has no <cstdint>, then the
// kernel header.
const char kPrelude[] =
    "typedef unsigned char uint8_t;\n"
    "typedef unsigned short uint16_t;\n"
    "typedef unsigned int uint32_t;\n"
    "typedef unsigned long long uint64_t;\n"
    "typedef signed char int8_t;\n"
    "typedef short int16_t;\n"
    "typedef int int32_t;\n"
    "typedef long long int64_t;\n";

// NVRTC is opened by path ($SBF_NVRTC_PATH, else the CUDA toolkit this
// library was built with) into its own namespace: a process may already hold
// another libnvrtc.so.12 (Python frameworks ship their own), and an older one
// rejects the tile kernel's 256-bit loads.
struct Nvrtc {
    decltype(&nvrtcVersion) version = nullptr;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcAddNameExpression) add_name = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcGetLoweredName) lowered = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    bool ok = false;
};

const Nvrtc& nvrtc() {
    static const Nvrtc api = [] {
        Nvrtc a;
        const char* env = std::getenv("SBF_NVRTC_PATH");
        const char* paths[] = {env, "/usr/local/cuda/lib64/libnvrtc.so.12",
                               "/usr/local/cuda/lib64/libnvrtc.so"};
        void* h = nullptr;
        for (const char* path : paths)
            if (path && (h = dlopen(path, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) return a;
        auto get = [&](auto& fn, const char* name) {
            fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
            return fn != nullptr;
        };
        a.ok = get(a.version, "nvrtcVersion") && get(a.create, "nvrtcCreateProgram") &&
               get(a.add_name, "nvrtcAddNameExpression") &&
               get(a.compile, "nvrtcCompileProgram") &&
               get(a.log_size, "nvrtcGetProgramLogSize") && get(a.log, "nvrtcGetProgramLog") &&
               get(a.cubin_size, "nvrtcGetCUBINSize") && get(a.cubin, "nvrtcGetCUBIN") &&
               get(a.lowered, "nvrtcGetLoweredName") && get(a.destroy, "nvrtcDestroyProgram");
        return a;
    }();
    return api;
}

// Kernel variants in KernelSet order: (query, dense, ragged).
constexpr bool kVariants[6][3] = {{false, false, false}, {true, false, false},
                                  {false, true, false},  {true, true, false},
                                  {false, false, true},  {true, false, true}};

uint64_t fnv1a(uint64_t h, const void* data, size_t n) {
    const auto* p = static_cast<const unsigned char*>(data);
    for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 0x100000001b3ULL;
    return h;
}

bool jit_enabled() {
    const char* v = std::getenv("SBF_JIT");
    return !(v && (std::strcmp(v, "0") == 0 || std::strcmp(v, "off") == 0));
}

std::string cache_dir() {
    if (const char* v = std::getenv("SBF_JIT_CACHE")) return v;
    if (const char* x = std::getenv("XDG_CACHE_HOME")) return std::string(x) + "/sbf_b200";
    if (const char* h = std::getenv("HOME")) return std::string(h) + "/.cache/sbf_b200";
    return "/tmp/sbf_b200_jit";
}

void make_dirs(const std::string& path) {
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

struct Compiled {
    std::vector<std::string> names;  // lowered kernel names, KernelSet order
    std::vector<char> cubin;
};

// One configuration to compile: DNA gets the tile kernels, other alphabets
// the generic kernels with the configuration as template constants.
struct JitConfig {
    int k, s, m, h, alphabet;
    uint32_t bits, width;
    bool tile() const { return alphabet == SBF_ALPHABET_DNA; }
};

std::string name_expr(const JitConfig& c, int v) {
    char cfg[96], buf[192];
    if (c.tile())
        std::snprintf(cfg, sizeof cfg, "sbf::tile_kernel<sbf::Cfg<%d, %d, %d, %d>", c.k, c.s, c.m,
                      c.h);
    else
        std::snprintf(cfg, sizeof cfg, "sbf::generic_kernel<sbf::FixedGen<%d, %d, %d, %d, %u, %u, %d>",
                      c.k, c.s, c.m, c.h, c.bits, c.width, c.alphabet);
    std::snprintf(buf, sizeof buf, "&%s, %s, %s, %s>", cfg, kVariants[v][0] ? "true" : "false",
                  kVariants[v][1] ? "true" : "false", kVariants[v][2] ? "true" : "false");
    return buf;
}

bool compile(const JitConfig& c, const std::string& arch, Compiled* out) {
    const Nvrtc& nv = nvrtc();
    if (!nv.ok) return false;
    const char* headers[] = {kJitInternal, kJitDevice, kJitFlush, kJitTile, kJitGeneric};
    const char* names[] = {"sbf_internal.h", "sbf_device.cuh", "sbf_flush.cuh", "sbf_tile.cuh",
                           "sbf_generic.cuh"};
    const std::string src = std::string(kPrelude) +
                            (c.tile() ? "#include \"sbf_tile.cuh\"\n" : "#include \"sbf_generic.cuh\"\n");
    nvrtcProgram prog;
    if (nv.create(&prog, src.c_str(), "sbf_jit.cu", 5, headers, names) != NVRTC_SUCCESS)
        return false;
    std::vector<std::string> exprs;
    for (int v = 0; v < 6; ++v) {
        exprs.push_back(name_expr(c, v));
        nv.add_name(prog, exprs.back().c_str());
    }
    const std::string arch_opt = "-arch=" + arch;
    const char* opts[] = {arch_opt.c_str(), "-std=c++17", "-lineinfo"};
    bool ok = nv.compile(prog, 3, opts) == NVRTC_SUCCESS;
    if (!ok && std::getenv("SBF_JIT_LOG")) {
        size_t n = 0;
        nv.log_size(prog, &n);
        std::string log(n, '\0');
        nv.log(prog, &log[0]);
        std::fprintf(stderr, "sbf_b200: run-time compilation failed:\n%s\n", log.c_str());
    }
    size_t size = 0;
    if (ok) ok = nv.cubin_size(prog, &size) == NVRTC_SUCCESS && size > 0;
    if (ok) {
        out->cubin.resize(size);
        ok = nv.cubin(prog, out->cubin.data()) == NVRTC_SUCCESS;
    }
    for (int v = 0; ok && v < 6; ++v) {
        const char* lowered = nullptr;
        ok = nv.lowered(prog, exprs[v].c_str(), &lowered) == NVRTC_SUCCESS && lowered;
        if (ok) out->names.push_back(lowered);
    }
    nv.destroy(&prog);
    return ok;
}

// Cache file: "SBFJIT1\n", six lowered names one per line, the cubin size
// on a line, then the cubin bytes.
bool read_cache(const std::string& path, Compiled* out) {
    std::ifstream in(path, std::ios::binary);
    if (!in) return false;
    std::string magic;
    if (!std::getline(in, magic) || magic != "SBFJIT1") return false;
    for (int v = 0; v < 6; ++v) {
        std::string n;
        if (!std::getline(in, n) || n.empty()) return false;
        out->names.push_back(n);
    }
    std::string size_line;
    if (!std::getline(in, size_line)) return false;
    const unsigned long long size = std::strtoull(size_line.c_str(), nullptr, 10);
    if (size == 0 || size > (256ull << 20)) return false;
    out->cubin.resize(size);
    in.read(out->cubin.data(), static_cast<std::streamsize>(size));
    return static_cast<unsigned long long>(in.gcount()) == size;
}

void write_cache(const std::string& dir, const std::string& path, const Compiled& c) {
    make_dirs(dir);
    const std::string tmp = path + ".tmp." + std::to_string(getpid());
    {
        std::ofstream out(tmp, std::ios::binary);
        if (!out) return;
        out << "SBFJIT1\n";
        for (const std::string& n : c.names) out << n << "\n";
        out << c.cubin.size() << "\n";
        out.write(c.cubin.data(), static_cast<std::streamsize>(c.cubin.size()));
        if (!out) return;
    }
    std::rename(tmp.c_str(), path.c_str());
}

struct JitEntry {
    KernelSet ks{};
    cudaLibrary_t lib = nullptr;
    std::set<int> devices;  // devices whose kernel attributes are set
};

std::mutex g_mu;
std::map<std::tuple<int, int, int, int, int>, std::unique_ptr<JitEntry>> g_sets;
std::set<std::tuple<int, int, int, int, int>> g_failed;

}  // namespace

const KernelSet* jit_kernels(int k, int s, int m, int h, int alphabet, int device) {
    if (!jit_enabled()) return nullptr;
    JitConfig jc{k, s, m, h, alphabet, 0, 0};
    if (!alphabet_geometry(alphabet, &jc.bits, &jc.width)) return nullptr;
    int major = 0, minor = 0;
    if (cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&minor, cudaDevAttrComputeCapabilityMinor, device) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    if (major != 10 || minor != 0) return nullptr;  // the library targets sm_100a
    const auto key = std::make_tuple(k, s, m, h, alphabet);
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_failed.count(key)) return nullptr;
    auto it = g_sets.find(key);
    if (it == g_sets.end()) {
        const std::string arch = "sm_100a";
        int nv_major = 0, nv_minor = 0;
        if (nvrtc().ok) nvrtc().version(&nv_major, &nv_minor);
        uint64_t hash = 0xcbf29ce484222325ULL;
        for (const char* src : {kJitInternal, kJitDevice, kJitFlush, kJitTile, kJitGeneric, kPrelude})
            hash = fnv1a(hash, src, std::strlen(src));
        const int meta[] = {k, s, m, h, alphabet, nv_major, nv_minor};
        hash = fnv1a(hash, meta, sizeof meta);
        hash = fnv1a(hash, arch.data(), arch.size());
        char file[128];
        std::snprintf(file, sizeof file, "%s_k%d_s%d_m%d_h%d_a%d_%016llx.bin",
                      jc.tile() ? "tile" : "generic", k, s, m, h, alphabet,
                      static_cast<unsigned long long>(hash));
        const std::string dir = cache_dir();
        const std::string path = dir + "/" + file;
        Compiled c;
        if (!read_cache(path, &c)) {
            c = Compiled{};
            if (!compile(jc, arch, &c)) {
                g_failed.insert(key);
                return nullptr;
            }
            write_cache(dir, path, c);
        }
        auto e = std::make_unique<JitEntry>();
        if (cudaLibraryLoadData(&e->lib, c.cubin.data(), nullptr, nullptr, 0, nullptr, nullptr,
                                0) != cudaSuccess) {
            cudaGetLastError();
            g_failed.insert(key);
            return nullptr;
        }
        const void* fns[6] = {};
        for (int v = 0; v < 6; ++v) {
            cudaKernel_t kern = nullptr;
            if (cudaLibraryGetKernel(&kern, e->lib, c.names[v].c_str()) != cudaSuccess) {
                cudaGetLastError();
                cudaLibraryUnload(e->lib);
                g_failed.insert(key);
                return nullptr;
            }
            fns[v] = reinterpret_cast<const void*>(kern);
        }
        e->ks = KernelSet{k, s, m, h, fns[0], fns[1], fns[2], fns[3], fns[4], fns[5]};
        e->ks.jit = true;
        if (!jc.tile()) {
            // The generic kernels use few registers; inserts take the flush
            // ring's dynamic shared memory, queries none.
            e->ks.smem_query = 0;
            e->ks.jit_occupancy = 4;
        }
        it = g_sets.emplace(key, std::move(e)).first;
    }
    JitEntry& e = *it->second;
    if (!e.devices.count(device)) {
        const void* fns[6] = {e.ks.insert_bytes, e.ks.query_bytes,   e.ks.insert_dense,
                              e.ks.query_dense,  e.ks.insert_ragged, e.ks.query_ragged};
        for (int v = 0; v < 6; ++v) {
            const int dyn = e.ks.smem(kVariants[v][0]);
            if (dyn == 0) continue;
            if (cudaKernelSetAttributeForDevice(
                    reinterpret_cast<cudaKernel_t>(const_cast<void*>(fns[v])),
                    cudaFuncAttributeMaxDynamicSharedMemorySize, dyn, device) != cudaSuccess) {
                cudaGetLastError();
                return nullptr;
            }
        }
        e.devices.insert(device);
    }
    return &e.ks;
}

}  // namespace sbf
