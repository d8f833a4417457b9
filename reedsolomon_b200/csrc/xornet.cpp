// xornet.cpp -- bit-sliced XOR-network kernels, generated per coefficient
// matrix and compiled at run time (NVRTC) for sm_100a.
//
// Multiplication by a constant c in GF(2^8) is linear over GF(2): the bits of
// c*x are fixed XORs of the bits of x (column a of the 8x8 bit matrix is
// c*2^a).  The reference exploits this on x86 with GFNI affine transforms
// (mulGFNI_*, galois_gen_amd64.s; the 8x8 matrices come from genGFNIMatrix,
// galois.go:1004-1016).  A coefficient tile of n_out x n_in bytes is thus one
// (8 n_out) x (8 n_in) bit matrix, and every output bit-plane is the XOR of a
// fixed set of input bit-planes.  The generated kernel:
//
//   * gives each warp 1 KiB of every shard per step: lane l loads the 16-byte
//     vectors l and l+32, i.e. eight 32-bit words w0..w7;
//   * transposes the eight words as 8x8 bit blocks (three delta-swap stages,
//     two shifts and two bit selects per swap), so word a becomes bit-plane a
//     of the lane's 32 bytes;
//   * XORs the planes into 8 n_out accumulator planes with a schedule fixed
//     at generation time: inputs are taken three at a time and common pairs of
//     planes are factored out greedily (Paar's heuristic), and the XOR chains
//     fuse into three-input LOP3s;
//   * issues every group's loads before the previous group is multiplied, and
//     the next chunk's first group before this chunk's last one;
//   * transposes the accumulators back and stores them (or XORs into the
//     outputs, or compares with them for verification).
//
// Per input byte of RS(10,4) this runs about 4.9 integer instructions (all
// on the ALU and FMA pipes) and no shared-memory lookups; the nibble-table
// kernel needs two lookups per byte and saturates the shared-memory pipe
// first.  Kernels are cached per (mode, n_in, n_out, coefficients); a matrix
// that is not compiled yet is queued for a background compile and the caller
// runs a table kernel meanwhile.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nvrtc.h>

#include <pthread.h>
#include <sys/stat.h>
#include <unistd.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

#include "gf_host.h"
#include "kernels.h"
#include "xornet.h"

namespace rsgpu {
namespace {

// ---- source generation ------------------------------------------------------

// Bits of c * 2^a for a = 0..7: bit b of column a is M[b][a].
uint8_t mul_column(uint8_t c, int a) { return gf_mul(c, (uint8_t)(1u << a)); }

struct Emitter {
    std::string s;
    void line(const std::string &x) {
        s += x;
        s += '\n';
    }
};

std::string plane_name(int i, int a) { return "p" + std::to_string(i) + "_" + std::to_string(a); }
std::string acc_name(int j, int b) { return "o" + std::to_string(j) + "_" + std::to_string(b); }

// Greedy pair factoring over the rows of one input group: while some pair of
// terms occurs in two or more rows, introduce t = x ^ y for the most frequent
// pair (ties: the lexicographically first) and substitute it.
void factor_pairs(std::vector<std::vector<int>> &rows, int &next_term, std::vector<std::pair<int, int>> &temps) {
    for (;;) {
        std::map<std::pair<int, int>, int> count;
        for (auto &r : rows)
            for (size_t u = 0; u < r.size(); u++)
                for (size_t v = u + 1; v < r.size(); v++) count[{r[u], r[v]}]++;
        std::pair<int, int> best{-1, -1};
        int best_n = 1;
        for (auto &kv : count)
            if (kv.second > best_n) {
                best_n = kv.second;
                best = kv.first;
            }
        if (best.first < 0) return;
        const int t = next_term++;
        temps.push_back(best);
        for (auto &r : rows) {
            auto x = std::find(r.begin(), r.end(), best.first);
            auto y = std::find(r.begin(), r.end(), best.second);
            if (x == r.end() || y == r.end()) continue;
            r.erase(std::remove_if(r.begin(), r.end(), [&](int e) { return e == best.first || e == best.second; }),
                    r.end());
            r.push_back(t);
            std::sort(r.begin(), r.end());
        }
    }
}

const char *kPreamble = R"(
typedef unsigned int u32;
struct XnArgs {
    const uint4 *in[32];
    uint4 *out[16];
    long long nchunk;
    int *flag;
};
// Exchanges bits mh = m << s of x with bits m of y (one delta swap).
#define XN_SWAP(x, y, m, mh, s) { const u32 xs_ = (x) >> (s), ys_ = (y) << (s); \
    x = ((x) & ~(mh)) | (ys_ & (mh)); y = ((y) & ~(m)) | (xs_ & (m)); }
// 8x8 bit transpose of every byte lane of w0..w7 (an involution).
#define XN_T8(w0, w1, w2, w3, w4, w5, w6, w7) { \
    XN_SWAP(w0, w4, 0x0F0F0F0Fu, 0xF0F0F0F0u, 4) XN_SWAP(w1, w5, 0x0F0F0F0Fu, 0xF0F0F0F0u, 4) \
    XN_SWAP(w2, w6, 0x0F0F0F0Fu, 0xF0F0F0F0u, 4) XN_SWAP(w3, w7, 0x0F0F0F0Fu, 0xF0F0F0F0u, 4) \
    XN_SWAP(w0, w2, 0x33333333u, 0xCCCCCCCCu, 2) XN_SWAP(w1, w3, 0x33333333u, 0xCCCCCCCCu, 2) \
    XN_SWAP(w4, w6, 0x33333333u, 0xCCCCCCCCu, 2) XN_SWAP(w5, w7, 0x33333333u, 0xCCCCCCCCu, 2) \
    XN_SWAP(w0, w1, 0x55555555u, 0xAAAAAAAAu, 1) XN_SWAP(w2, w3, 0x55555555u, 0xAAAAAAAAu, 1) \
    XN_SWAP(w4, w5, 0x55555555u, 0xAAAAAAAAu, 1) XN_SWAP(w6, w7, 0x55555555u, 0xAAAAAAAAu, 1) }
)";

}  // namespace

std::string xornet_body(const uint8_t *coef, int stride, int n_in, int n_out, int mode, int group) {
    // The body is the whole chunk loop: XN_FIRST, XN_STRIDE, XN_N and XN_LANE
    // come from the wrapper, XN_LD(i, v) / XN_LDO(j, v) load 16-byte vector v
    // of input i / output j and XN_ST(j, v, x) stores it.  Each group's loads
    // are issued before the previous group is multiplied, the first group of
    // the next chunk and (xor / verify) this chunk's outputs before the last
    // group of this one.
    Emitter e;
    const int grp = group > 0 ? group : xornet_group(n_out);
    std::vector<std::pair<int, int>> groups;
    for (int g0 = 0; g0 < n_in; g0 += grp) groups.push_back({g0, std::min(n_in, g0 + grp)});
    auto qname = [](int i, char h) { return "q" + std::to_string(i) + h; };
    auto load = [&](int i, const char *v0, const char *v1, bool decl) {
        e.line(std::string(decl ? "const uint4 " : "") + qname(i, 'a') + " = XN_LD(" + std::to_string(i) + ", " + v0 +
               ")" + (decl ? ", " : "; ") + qname(i, 'b') + " = XN_LD(" + std::to_string(i) + ", " + v1 + ");");
    };
    e.line("long long c = XN_FIRST;");
    {
        std::string d = "uint4 ";
        for (int i = groups[0].first; i < groups[0].second; i++)
            d += qname(i, 'a') + ", " + qname(i, 'b') + (i + 1 < groups[0].second ? ", " : ";");
        e.line(d);
        e.line("if (c < XN_N) {");
        e.line("const long long v0 = c * 64 + XN_LANE, v1 = v0 + 32;");
        for (int i = groups[0].first; i < groups[0].second; i++) load(i, "v0", "v1", false);
        e.line("}");
    }
    e.line("for (; c < XN_N; c += XN_STRIDE) {");
    e.line("const long long v0 = c * 64 + XN_LANE, v1 = v0 + 32;");
    e.line("const long long n0 = (c + XN_STRIDE) * 64 + XN_LANE, n1 = n0 + 32;");
    e.line("const int more = c + XN_STRIDE < XN_N;");
    e.line("(void)n0; (void)n1; (void)more;");
    for (int j = 0; j < n_out; j++)
        for (int b = 0; b < 8; b++) e.line("u32 " + acc_name(j, b) + " = 0;");
    int next_term = 0;  // global temp numbering
    for (size_t gi = 0; gi < groups.size(); gi++) {
        const int g0 = groups[gi].first, g1 = groups[gi].second;
        for (int i = g0; i < g1; i++) {
            std::string decl = "u32 ";
            const char *f[8] = {"a.x", "a.y", "a.z", "a.w", "b.x", "b.y", "b.z", "b.w"};
            for (int a = 0; a < 8; a++)
                decl += plane_name(i, a) + " = q" + std::to_string(i) + f[a] + (a < 7 ? ", " : ";");
            e.line(decl);
        }
        if (gi + 1 < groups.size()) {
            for (int i = groups[gi + 1].first; i < groups[gi + 1].second; i++) load(i, "v0", "v1", true);
        } else {
            if (mode != kModeWrite)
                for (int j = 0; j < n_out; j++)
                    e.line("const uint4 e" + std::to_string(j) + "a = XN_LDO(" + std::to_string(j) + ", v0), e" +
                           std::to_string(j) + "b = XN_LDO(" + std::to_string(j) + ", v1);");
            e.line("if (more) {");
            for (int i = groups[0].first; i < groups[0].second; i++) load(i, "n0", "n1", false);
            e.line("}");
        }
        for (int i = g0; i < g1; i++) {
            std::string t = "XN_T8(";
            for (int a = 0; a < 8; a++) t += plane_name(i, a) + (a < 7 ? ", " : ")");
            e.line(t);
        }
        // Terms 0 .. 8*(g1-g0)-1 are the group's planes; later ids are temps.
        const int nplanes = 8 * (g1 - g0);
        std::vector<std::vector<int>> rows((size_t)8 * n_out);
        for (int j = 0; j < n_out; j++)
            for (int i = g0; i < g1; i++) {
                const uint8_t c = coef[(size_t)j * stride + i];
                for (int a = 0; a < 8; a++) {
                    const uint8_t col = mul_column(c, a);
                    for (int b = 0; b < 8; b++)
                        if ((col >> b) & 1) rows[(size_t)8 * j + b].push_back(8 * (i - g0) + a);
                }
            }
        for (auto &r : rows) std::sort(r.begin(), r.end());
        int local = nplanes;
        std::vector<std::pair<int, int>> temps;
        factor_pairs(rows, local, temps);
        auto name = [&](int id) {
            if (id < nplanes) return plane_name(g0 + id / 8, id % 8);
            return "t" + std::to_string(next_term + id - nplanes);
        };
        for (size_t u = 0; u < temps.size(); u++)
            e.line("const u32 " + name(nplanes + (int)u) + " = " + name(temps[u].first) + " ^ " +
                   name(temps[u].second) + ";");
        for (int j = 0; j < n_out; j++)
            for (int b = 0; b < 8; b++) {
                const auto &r = rows[(size_t)8 * j + b];
                if (r.empty()) continue;
                // One XOR chain per row; ptxas fuses it into three-input
                // LOP3s (forcing them by inline PTX serialises the chain and spills).
                std::string x = acc_name(j, b) + " ^= ";
                for (size_t w = 0; w < r.size(); w++) x += name(r[w]) + (w + 1 < r.size() ? " ^ " : ";");
                e.line(x);
            }
        next_term += local - nplanes;
    }
    for (int j = 0; j < n_out; j++) {
        std::string t = "XN_T8(";
        for (int b = 0; b < 8; b++) t += acc_name(j, b) + (b < 7 ? ", " : ")");
        e.line(t);
        const std::string J = std::to_string(j);
        auto o = [&](int b) { return acc_name(j, b); };
        const char *f[4] = {".x", ".y", ".z", ".w"};
        if (mode == kModeVerify) {
            std::string d = "diff |= ";
            for (int b = 0; b < 8; b++)
                d += "(" + o(b) + " ^ e" + J + (b < 4 ? "a" : "b") + f[b & 3] + ")" + (b < 7 ? " | " : ";");
            e.line(d);
            continue;
        }
        for (int h = 0; h < 2; h++) {
            std::string v = "make_uint4(";
            for (int b = 4 * h; b < 4 * h + 4; b++) {
                v += o(b);
                if (mode == kModeXor) v += " ^ e" + J + (h ? "b" : "a") + f[b & 3];
                v += (b & 3) == 3 ? ")" : ", ";
            }
            e.line("XN_ST(" + J + ", " + (h ? "v1" : "v0") + ", " + v + ");");
        }
    }
    e.line("}");
    return e.s;
}

int xornet_threads(int n_out) { return n_out <= 6 ? 512 : 256; }

int xornet_group(int n_out) { return n_out <= 6 ? 3 : 2; }

std::string xornet_source(const uint8_t *coef, int stride, int n_in, int n_out, int mode, int group) {
    std::string s = "#define XN_THREADS " + std::to_string(xornet_threads(n_out)) + "\n";
    s += kPreamble;
    s += R"(
#define XN_LD(i, v) __ldcs(a.in[i] + (v))
#define XN_LDO(j, v) __ldcs(a.out[j] + (v))
#define XN_ST(j, v, x) __stcs(a.out[j] + (v), x)
// One CTA per SM by design: without the minimum, ptxas may aim at full
// occupancy (32 registers) and spill most of the network.
extern "C" __global__ void __launch_bounds__(XN_THREADS, 1) rs_xornet(const __grid_constant__ XnArgs a) {
    const long long XN_STRIDE = ((long long)gridDim.x * blockDim.x) >> 5;
    const long long XN_FIRST = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const long long XN_LANE = threadIdx.x & 31, XN_N = a.nchunk;
    u32 diff = 0;
)";
    s += xornet_body(coef, stride, n_in, n_out, mode, group);
    s += R"(    if (diff) *a.flag = 1;
}
)";
    return s;
}

std::string xornet_host_source(const uint8_t *coef, int stride, int n_in, int n_out, int mode, int group) {
    std::string s = R"(#include <stdint.h>
typedef struct { unsigned x, y, z, w; } uint4;
static inline uint4 make_uint4(unsigned x, unsigned y, unsigned z, unsigned w) { uint4 r = {x, y, z, w}; return r; }
)";
    s += kPreamble;
    s += R"(
#define XN_LD(i, v) in[i][v]
#define XN_LDO(j, v) out[j][v]
#define XN_ST(j, v, x) (out[j][v] = (x))
void rs_xornet_host(const uint4 *const *in, uint4 *const *out, long long nchunk, int *flag) {
    u32 diff = 0;
    const long long XN_FIRST = 0, XN_STRIDE = 1, XN_N = nchunk;
    for (long long XN_LANE = 0; XN_LANE < 32; XN_LANE++) {
)";
    s += xornet_body(coef, stride, n_in, n_out, mode, group);
    s += R"(    }
    if (diff) *flag = 1;
}
)";
    return s;
}

namespace {

// ---- NVRTC (loaded on first use; absent => no XOR-network kernels) ----------

struct Nvrtc {
    bool ok = false;
    decltype(&nvrtcCreateProgram) create = nullptr;
    decltype(&nvrtcCompileProgram) compile = nullptr;
    decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
    decltype(&nvrtcGetCUBIN) cubin = nullptr;
    decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
    decltype(&nvrtcGetProgramLog) log = nullptr;
    decltype(&nvrtcDestroyProgram) destroy = nullptr;
    int major = 0, minor = 0;  // nvrtcVersion, part of the on-disk cache key
    Nvrtc() {
        // RSGPU_NVRTC: a path to load instead, or "off" (no XOR-network kernels).
        const char *env = getenv("RSGPU_NVRTC");
        if (env && strcmp(env, "off") == 0) return;
        const char *names[] = {env, "libnvrtc.so.12", "libnvrtc.so"};
        void *h = nullptr;
        for (const char *n : names)
            if (n && *n && (h = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
        if (!h) return;
        create = (decltype(create))dlsym(h, "nvrtcCreateProgram");
        compile = (decltype(compile))dlsym(h, "nvrtcCompileProgram");
        cubin_size = (decltype(cubin_size))dlsym(h, "nvrtcGetCUBINSize");
        cubin = (decltype(cubin))dlsym(h, "nvrtcGetCUBIN");
        log_size = (decltype(log_size))dlsym(h, "nvrtcGetProgramLogSize");
        log = (decltype(log))dlsym(h, "nvrtcGetProgramLog");
        destroy = (decltype(destroy))dlsym(h, "nvrtcDestroyProgram");
        ok = create && compile && cubin_size && cubin && log_size && log && destroy;
        auto version = (decltype(&nvrtcVersion))dlsym(h, "nvrtcVersion");
        if (version) version(&major, &minor);
    }
};

const Nvrtc &nvrtc() {
    static const Nvrtc *n = new Nvrtc();  // never destroyed: the worker may outlive static teardown
    return *n;
}

// Compiles one generated kernel to an sm_100a cubin; empty on failure.
// *spill receives the spill-store bytes ptxas reports (-1 if unknown).  The
// log goes to stderr on failure when RSGPU_XORNET_LOG is set.
std::atomic<int> g_compiles{0};  // NVRTC compilations in this process

std::vector<char> compile_cubin(const std::string &src, int *spill) {
    const Nvrtc &nv = nvrtc();
    std::vector<char> out;
    *spill = -1;
    if (!nv.ok) return out;
    g_compiles++;
    nvrtcProgram prog;
    if (nv.create(&prog, src.c_str(), "rs_xornet.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS) return out;
    const char *opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device", "--ptxas-options=-v"};
    const nvrtcResult rc = nv.compile(prog, 4, opts);
    size_t n = 0;
    nv.log_size(prog, &n);
    std::string log(n, '\0');
    if (n) nv.log(prog, &log[0]);
    if (rc == NVRTC_SUCCESS) {
        size_t m = 0;
        if (nv.cubin_size(prog, &m) == NVRTC_SUCCESS && m) {
            out.resize(m);
            if (nv.cubin(prog, out.data()) != NVRTC_SUCCESS) out.clear();
        }
        const size_t at = log.find(" bytes spill stores");
        if (at != std::string::npos) {
            size_t b = at;
            while (b > 0 && isdigit((unsigned char)log[b - 1])) b--;
            *spill = atoi(log.c_str() + b);
        }
    } else if (getenv("RSGPU_XORNET_LOG")) {
        fprintf(stderr, "rs_xornet compile failed:\n%s\n", log.c_str());
    }
    nv.destroy(&prog);
    return out;
}

// ---- cache ---------------------------------------------------------------------

struct Key {
    int n_in, n_out, mode;
    std::vector<uint8_t> coef;  // n_out x n_in, row-major
    bool operator<(const Key &o) const {
        if (mode != o.mode) return mode < o.mode;
        if (n_in != o.n_in) return n_in < o.n_in;
        if (n_out != o.n_out) return n_out < o.n_out;
        return coef < o.coef;
    }
};

struct Entry {
    // kQueued: waiting in the queue; kCompiling: a worker or a synchronous
    // caller is compiling it; kCompiled / kFailed: final.
    enum State { kQueued, kCompiling, kCompiled, kFailed } state = kQueued;
    bool final_state() const { return state == kCompiled || state == kFailed; }
    std::vector<char> cubin;
    cudaLibrary_t lib = nullptr;
    cudaKernel_t kern = nullptr;
    int blocks_per_sm[64][5] = {};  // [device ordinal][log2 warps per CTA], 0 = not queried
    // Eviction bookkeeping (all under the cache lock): the cache clock at the
    // last lookup; launches between their lookup and the event recorded
    // behind them; events (device, event) recorded behind launches that may
    // still run, one per launch; and whether a launch was captured into a
    // graph (then the library is never unloaded).
    uint64_t last_use = 0;
    int launching = 0;
    std::vector<std::pair<int, cudaEvent_t>> pending;
    bool pinned = false;
};

struct Cache {
    std::mutex mu;
    std::condition_variable cv, idle;
    std::map<Key, std::shared_ptr<Entry>> map;
    std::deque<std::pair<Key, std::shared_ptr<Entry>>> queue;
    int workers = 0;
    int busy = 0;
    uint64_t clock = 0;
    std::map<Key, int> uses;  // launches of matrices not compiled yet (bounded)
    std::vector<cudaEvent_t> free_events[64];  // per device, completed and reusable
};

// A matrix is compiled (in the background) once this many launches have
// asked for it: one-off matrices (a decode matrix seen once) are not worth a
// compile of 0.2-5 s and a module.  RSGPU_XORNET_MIN_USES overrides it (1:
// compile on first sight).
int min_uses() {
    static const int n = [] {
        const char *e = getenv("RSGPU_XORNET_MIN_USES");
        const int v = e ? atoi(e) : 2;
        return v < 1 ? 1 : v;
    }();
    return n;
}
constexpr size_t kUsesCap = 16384;  // matrices counted before the counts are reset

// Entries kept (kXornetCacheCap; RSGPU_XORNET_CACHE_CAP overrides it): past
// it, the least recently used idle entry is evicted and its library unloaded.
size_t cache_cap() {
    static const size_t n = [] {
        const char *e = getenv("RSGPU_XORNET_CACHE_CAP");
        const long v = e ? atol(e) : kXornetCacheCap;
        return (size_t)(v < 1 ? 1 : v);
    }();
    return n;
}

void worker_loop();
Cache &cache();
void drain_at_exit();

// Starts a compile worker when queued work has no free one, up to a quarter
// of the host threads (1..4).  Workers never exit (the queue and the cache
// outlive static teardown).  Called with the cache lock held.
void spawn_workers_locked(Cache &c) {
    const int cap = std::max(1, std::min(4, (int)std::thread::hardware_concurrency() / 4));
    if (!c.queue.empty() && c.workers < cap && c.busy == c.workers) {
        // Before the first worker starts: drain at exit through atexit.  NVRTC
        // is loaded (dlopen) after this library, so its static destructors
        // run before this library's; a handler registered now runs before
        // them, while no worker may still be inside NVRTC.
        static std::once_flag registered;
        std::call_once(registered, [] { std::atexit(drain_at_exit); });
        std::thread(worker_loop).detach();
        c.workers++;
    }
}

// fork(): the child inherits none of the worker threads.  The lock is held
// across fork so the child's copy of the cache is consistent; the child then
// forgets the workers, puts back in the queue the matrices that were being
// compiled, and starts workers on demand (the next queued compile or wait),
// not from the handler.  Condition variables are rebuilt: no thread waits
// on them in the child.
void fork_prepare() { cache().mu.lock(); }
void fork_parent() { cache().mu.unlock(); }
void fork_child() {
    Cache &c = cache();
    new (&c.cv) std::condition_variable();
    new (&c.idle) std::condition_variable();
    c.workers = 0;
    c.busy = 0;
    for (auto &kv : c.map)
        if (kv.second->state == Entry::kCompiling) {
            kv.second->state = Entry::kQueued;
            c.queue.emplace_back(kv.first, kv.second);
        }
    c.mu.unlock();
}

Cache &cache() {
    static Cache *c = [] {
        Cache *p = new Cache();  // never destroyed (see nvrtc())
        pthread_atfork(fork_prepare, fork_parent, fork_child);
        return p;
    }();
    return *c;
}

// Register pressure of the straight-line network decides the factoring
// group: the preferred size first, then smaller ones, keeping the first
// kernel that spills at most kSpillOk bytes (else the one that spills least).
constexpr int kSpillOk = 128;

// ---- optional on-disk cache --------------------------------------------------
// RSGPU_KERNEL_CACHE=<directory> keeps every final cubin in a file named by a
// 64-bit FNV-1a hash of the kernel's generated source (preferred group), the
// NVRTC version and the target, so a new process loads it instead of
// compiling.  A file is used only when its header (magic, source hash, size)
// matches and the cubin bytes hash to the value stored beside them, so a
// truncated or bit-flipped file is recompiled rather than run.  The hash is
// a corruption check, not an authentication: whoever can write the directory
// can make this process run their code, so it must be a directory only the
// library's user can write (it is created with mode 0700).  Files are
// written to a temporary name and renamed into place.
struct DiskHeader {
    char magic[8];
    uint64_t hash;       // of the generated source, NVRTC version and target
    uint64_t size;       // cubin bytes that follow
    uint64_t body_hash;  // of those bytes
};
constexpr char kDiskMagic[8] = {'R', 'S', 'X', 'N', 'C', '0', '2', '\0'};
constexpr uint64_t kDiskMaxBytes = 64ull << 20;

uint64_t fnv1a(const char *p, size_t n) {
    uint64_t h = 0xcbf29ce484222325ull;
    for (size_t i = 0; i < n; i++) {
        h ^= (unsigned char)p[i];
        h *= 0x100000001b3ull;
    }
    return h;
}
uint64_t fnv1a(const std::string &s) { return fnv1a(s.data(), s.size()); }

bool disk_read(const std::string &path, uint64_t hash, std::vector<char> &out) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    DiskHeader h;
    bool ok = fread(&h, sizeof h, 1, f) == 1 && memcmp(h.magic, kDiskMagic, sizeof kDiskMagic) == 0 &&
              h.hash == hash && h.size > 0 && h.size <= kDiskMaxBytes;
    if (ok) {
        out.resize(h.size);
        ok = fread(out.data(), 1, h.size, f) == h.size && fgetc(f) == EOF &&
             fnv1a(out.data(), out.size()) == h.body_hash;
    }
    fclose(f);
    if (!ok) out.clear();
    return ok;
}

void disk_write(const std::string &dir, const std::string &path, uint64_t hash, const std::vector<char> &bin) {
    static std::atomic<unsigned> seq{0};
    mkdir(dir.c_str(), 0700);  // one level; an existing directory is used as it is
    const std::string tmp = path + ".tmp." + std::to_string((long)getpid()) + "." + std::to_string(seq++);
    FILE *f = fopen(tmp.c_str(), "wb");
    if (!f) return;
    DiskHeader h;
    memcpy(h.magic, kDiskMagic, sizeof kDiskMagic);
    h.hash = hash;
    h.size = bin.size();
    h.body_hash = fnv1a(bin.data(), bin.size());
    const bool ok = fwrite(&h, sizeof h, 1, f) == 1 && fwrite(bin.data(), 1, bin.size(), f) == bin.size();
    if (fclose(f) == 0 && ok) rename(tmp.c_str(), path.c_str());
    else remove(tmp.c_str());
}

std::vector<char> build_kernel(const Key &k) {
    const char *dir_env = getenv("RSGPU_KERNEL_CACHE");
    const std::string dir = dir_env ? dir_env : "";
    std::string path;
    uint64_t hash = 0;
    if (!dir.empty()) {
        const Nvrtc &nv = nvrtc();
        hash = fnv1a(xornet_source(k.coef.data(), k.n_in, k.n_in, k.n_out, k.mode, xornet_group(k.n_out)) +
                     "|nvrtc " + std::to_string(nv.major) + "." + std::to_string(nv.minor) + "|sm_100a");
        char name[48];
        snprintf(name, sizeof name, "/rs_xornet_%016llx.cubin", (unsigned long long)hash);
        path = dir + name;
        std::vector<char> cached;
        if (disk_read(path, hash, cached)) return cached;
    }
    std::vector<char> best;
    int best_spill = 1 << 30;
    for (int g = xornet_group(k.n_out); g >= 1; g--) {
        int spill = 0;
        std::vector<char> bin = compile_cubin(xornet_source(k.coef.data(), k.n_in, k.n_in, k.n_out, k.mode, g), &spill);
        if (bin.empty()) continue;
        if (spill < 0) spill = 0;
        if (spill < best_spill) {
            best = std::move(bin);
            best_spill = spill;
        }
        if (best_spill <= kSpillOk) break;
    }
    if (!path.empty() && !best.empty()) disk_write(dir, path, hash, best);
    return best;
}

void worker_loop() {
    Cache &c = cache();
    for (;;) {
        std::pair<Key, std::shared_ptr<Entry>> job;
        {
            std::unique_lock<std::mutex> lk(c.mu);
            c.cv.wait(lk, [&] { return !c.queue.empty(); });
            job = std::move(c.queue.front());
            c.queue.pop_front();
            job.second->state = Entry::kCompiling;
            c.busy++;
        }
        std::vector<char> bin = build_kernel(job.first);
        // NVRTC registers exit handlers of its own during its first compile
        // (function-local statics); handlers run in reverse order, so the
        // drain is registered once more after that, to run before them.
        static std::once_flag after_first;
        std::call_once(after_first, [] { std::atexit(drain_at_exit); });
        {
            std::lock_guard<std::mutex> lk(c.mu);
            job.second->cubin = std::move(bin);
            job.second->state = job.second->cubin.empty() ? Entry::kFailed : Entry::kCompiled;
            c.busy--;
        }
        c.idle.notify_all();
    }
}

// At exit (atexit, registered when the first worker starts and again after
// the first compile; and at library unload) queued compiles are dropped and
// a compile in progress is waited for (bounded), so no worker is inside
// NVRTC while the process tears down.  A compile that is still in NVRTC's
// first run when exit starts can meet handlers NVRTC registered during that
// run, which run first; hosts that may exit with compiles in flight call
// rsgpu_xornet_drain() before exiting (the Python package does, through
// atexit, which runs before any of the C-level teardown).
void drain_at_exit() {
    Cache &c = cache();
    std::unique_lock<std::mutex> lk(c.mu);
    for (auto &q : c.queue) q.second->state = Entry::kFailed;
    c.queue.clear();
    c.idle.notify_all();  // waiters for an empty queue
    c.idle.wait_for(lk, std::chrono::seconds(30), [&] { return c.busy == 0; });
}
struct DrainAtExit {
    ~DrainAtExit() { drain_at_exit(); }
} g_drain_at_exit;

Key make_key(const GfMatArgs &a, int mode) {
    Key k;
    k.mode = mode;
    k.n_in = a.n_in;
    k.n_out = a.n_out;
    k.coef.resize((size_t)a.n_in * a.n_out);
    for (int o = 0; o < a.n_out; o++)
        for (int i = 0; i < a.n_in; i++) k.coef[(size_t)o * a.n_in + i] = a.coef[o][i];
    return k;
}

// Unloads evicted entries: waits (per device) for the event recorded after
// each one's last launch, then unloads its library.  Called without the lock.
void unload(std::vector<std::shared_ptr<Entry>> &victims) {
    for (auto &v : victims) {
        for (auto &pe : v->pending) {
            cudaEventSynchronize(pe.second);
            cudaEventDestroy(pe.second);
        }
        v->pending.clear();
        if (v->lib) cudaLibraryUnload(v->lib);
    }
    victims.clear();
}

// An event for a launch on device d: a pooled one, or a new one.  Events
// behind this entry's earlier launches that have completed go back to the
// pool first.  Called with the lock.
cudaEvent_t launch_event_locked(Cache &c, Entry &e, int d) {
    for (size_t i = 0; i < e.pending.size();) {
        if (cudaEventQuery(e.pending[i].second) == cudaSuccess) {
            c.free_events[e.pending[i].first].push_back(e.pending[i].second);
            e.pending[i] = e.pending.back();
            e.pending.pop_back();
        } else {
            i++;
        }
    }
    cudaEvent_t ev = nullptr;
    if (!c.free_events[d].empty()) {
        ev = c.free_events[d].back();
        c.free_events[d].pop_back();
    } else if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
        return nullptr;
    }
    return ev;
}

// Makes room for one entry when the cache is full: evicts the least recently
// used final entry that no launch is using and no graph holds.  False when
// every entry is busy, queued, compiling or pinned.  Called with the lock.
bool evict_one_locked(Cache &c, std::vector<std::shared_ptr<Entry>> &victims) {
    auto best = c.map.end();
    for (auto it = c.map.begin(); it != c.map.end(); ++it) {
        const Entry &e = *it->second;
        if (!e.final_state() || e.launching > 0 || e.pinned) continue;
        if (best == c.map.end() || e.last_use < best->second->last_use) best = it;
    }
    if (best == c.map.end()) return false;
    victims.push_back(best->second);
    c.map.erase(best);
    return true;
}

// The compiled entry for a's coefficients: compiles now when `sync`, else
// queues a background compile (once the matrix has been asked for
// min_uses() times) and returns null until it is ready.  `launch`: the caller
// launches it, and releases it with launch_done() after recording its event.
std::shared_ptr<Entry> lookup(const GfMatArgs &a, int mode, bool sync, bool launch = false) {
    if (!nvrtc().ok) return nullptr;
    Cache &c = cache();
    Key key = make_key(a, mode);
    std::shared_ptr<Entry> e;
    std::vector<std::shared_ptr<Entry>> victims;
    {
        std::unique_lock<std::mutex> lk(c.mu);
        auto it = c.map.find(key);
        if (it != c.map.end()) {
            e = it->second;
            e->last_use = ++c.clock;
            if (e->state == Entry::kCompiled) {
                if (launch) e->launching++;
                return e;
            }
            if (e->state == Entry::kFailed || !sync) return nullptr;
            if (e->state == Entry::kCompiling) {
                // someone else is compiling this entry: wait for them
                c.idle.wait(lk, [&] { return e->final_state(); });
                if (e->state != Entry::kCompiled) return nullptr;
                if (launch) e->launching++;
                return e;
            }
            // still queued: take it out of the queue and compile it here
            for (auto q = c.queue.begin(); q != c.queue.end(); ++q)
                if (q->second == e) {
                    c.queue.erase(q);
                    break;
                }
        } else {
            if (!sync) {
                if (c.uses.size() >= kUsesCap) c.uses.clear();
                if (++c.uses[key] < min_uses()) return nullptr;
                c.uses.erase(key);
            }
            if (c.map.size() >= cache_cap() && !evict_one_locked(c, victims)) return nullptr;
            e = std::make_shared<Entry>();
            e->last_use = ++c.clock;
            c.map.emplace(key, e);
            if (!sync) {
                c.queue.emplace_back(key, e);
                spawn_workers_locked(c);
                c.cv.notify_one();
                lk.unlock();
                unload(victims);
                return nullptr;
            }
        }
        e->state = Entry::kCompiling;
    }
    unload(victims);
    std::vector<char> bin = build_kernel(key);
    {
        std::lock_guard<std::mutex> lk(c.mu);
        e->cubin = std::move(bin);
        e->state = e->cubin.empty() ? Entry::kFailed : Entry::kCompiled;
        if (launch && e->state == Entry::kCompiled) e->launching++;
    }
    c.idle.notify_all();
    return e->state == Entry::kCompiled ? e : nullptr;
}

// Host mirror of XnArgs in the generated source (same member order and types).
struct XnArgs {
    const void *in[32];
    void *out[16];
    long long nchunk;
    int *flag;
};

}  // namespace

bool xornet_available() { return nvrtc().ok; }

int xornet_compile_count() { return g_compiles.load(); }

void xornet_drain() { drain_at_exit(); }

bool xornet_prepare(const GfMatArgs &a, int mode) {
    return a.n_in <= 32 && a.n_out <= kXornetMaxOut && lookup(a, mode, true) != nullptr;
}

int xornet_wait_idle() {
    Cache &c = cache();
    std::unique_lock<std::mutex> lk(c.mu);
    spawn_workers_locked(c);  // queued work without workers (a forked child)
    c.cv.notify_all();
    c.idle.wait(lk, [&] { return c.queue.empty() && c.busy == 0; });
    int n = 0;
    for (auto &kv : c.map) n += kv.second->state == Entry::kCompiled;
    return n;
}

cudaError_t xornet_launch(cudaStream_t st, const DeviceInfo &dev, const GfMatArgs &a, int mode, bool sync,
                          long long *bytes_done) {
    *bytes_done = 0;
    const long long nchunk = a.nbytes / kXornetChunk;
    if (nchunk == 0 || a.n_in > 32 || a.n_out > kXornetMaxOut) return cudaSuccess;
    for (int i = 0; i < a.n_in; i++)
        if (reinterpret_cast<uintptr_t>(a.in[i]) & 15u) return cudaSuccess;
    for (int o = 0; o < a.n_out; o++)
        if (reinterpret_cast<uintptr_t>(a.out[o]) & 15u) return cudaSuccess;
    std::shared_ptr<Entry> e = lookup(a, mode, sync, /*launch=*/true);
    if (!e) return cudaSuccess;
    Cache &c = cache();
    // Warps per CTA: the compiled maximum, halved while that would leave SMs
    // without work (1 MiB shards are 1024 warp steps: 4-warp CTAs spread
    // them over every SM where 16-warp CTAs would fill 64).
    int lw = 0;
    while ((32 << (lw + 1)) <= xornet_threads(a.n_out)) lw++;
    while (lw > 0 && nchunk < (long long)dev.sm_count << lw) lw--;
    const int threads = 32 << lw;
    const int d = dev.device & 63;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(st, &cap) != cudaSuccess) cap = cudaStreamCaptureStatusInvalidated;
    const bool capturing = cap != cudaStreamCaptureStatusNone;
    cudaKernel_t kern;
    int nb;
    {
        std::lock_guard<std::mutex> lk(c.mu);
        if (!e->lib) {
            // No module loading inside a stream capture: the table kernel
            // stands in until an uncaptured launch has loaded this one.
            if (capturing) {
                e->launching--;
                return cudaSuccess;
            }
            cudaError_t rc = cudaLibraryLoadData(&e->lib, e->cubin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0);
            if (rc == cudaSuccess) rc = cudaLibraryGetKernel(&e->kern, e->lib, "rs_xornet");
            if (rc != cudaSuccess) {
                e->launching--;
                return rc;
            }
        }
        // A graph holding this kernel may be replayed at any time: never
        // unload it once a launch has been captured.
        if (capturing) e->pinned = true;
        kern = e->kern;
        int &slot = e->blocks_per_sm[d][lw];
        if (slot == 0) {
            int q = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&q, (const void *)kern, threads, 0) !=
                    cudaSuccess ||
                q < 1)
                q = 1;
            slot = q;
        }
        nb = slot;
    }
    XnArgs x;
    memset(&x, 0, sizeof(x));
    for (int i = 0; i < a.n_in; i++) x.in[i] = a.in[i];
    for (int o = 0; o < a.n_out; o++) x.out[o] = a.out[o];
    x.nchunk = nchunk;
    x.flag = a.flag;
    const long long warps_per_cta = threads / 32;
    const long long want = (nchunk + warps_per_cta - 1) / warps_per_cta;
    const int grid = (int)std::max(1LL, std::min(want, (long long)dev.sm_count * nb));
    void *args[] = {&x};
    cudaError_t rc = cudaLaunchKernel((const void *)kern, dim3(grid), dim3(threads), args, 0, st);
    {
        // the event an eviction waits for before unloading the library
        std::lock_guard<std::mutex> lk(c.mu);
        if (rc == cudaSuccess && !capturing) {
            cudaEvent_t ev = launch_event_locked(c, *e, d);
            if (!ev) {
                e->pinned = true;  // nothing to wait on: keep the library for good
            } else if (cudaEventRecord(ev, st) != cudaSuccess) {
                cudaEventDestroy(ev);
                e->pinned = true;
            } else {
                e->pending.emplace_back(d, ev);
            }
        }
        e->launching--;
    }
    if (rc == cudaSuccess) *bytes_done = nchunk * kXornetChunk;
    return rc;
}

}  // namespace rsgpu
