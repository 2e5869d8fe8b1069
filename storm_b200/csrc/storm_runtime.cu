// Host runtime of the C ABI (include/storm_cuda.h): handle lifecycle, device
// memory, the order of kernels in a time step, and state transfer.  One CUDA
// stream per handle; every kernel launch goes through this file.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "storm_cuda.h"
#include "storm_internal.h"

using namespace storm;

namespace {

template <class T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0;
};

struct BankBuf {
    Bank b{};
    size_t cap = 0;
};

}  // namespace

struct StormHandle {
    StormProblemDesc desc{};
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t evStart = nullptr, evTransport0 = nullptr, evTransport1 = nullptr, evEnd = nullptr;
    cudaEvent_t evAfterEmit = nullptr, evAfterComb = nullptr;
    // storm_cuda_step_host: the census upload's own stream and its events
    cudaStream_t copyStream = nullptr;
    cudaEvent_t evCopyGo = nullptr, evCells = nullptr;
    std::vector<cudaEvent_t> evChunks;   // one per census chunk in place
    unsigned char *pinned = nullptr;   // the stream set's page-locked readback buffer (kPinnedBytes)
    uint32_t nx = 0, ny = 0, nz = 0, N = 0;
    std::vector<double> hxe, hye, hze, hxc, hyc, hzc;
    // device mesh + cells
    double *xe = nullptr, *ye = nullptr, *ze = nullptr, *xc = nullptr, *yc = nullptr, *zc = nullptr;
    float *hx = nullptr, *hy = nullptr, *hz = nullptr;   // FP32-tracking half widths
    bool fp32 = false;
    CellArrays A{};
    double *tabA = nullptr, *tabS = nullptr, *rhoF = nullptr;
    uint32_t *segs = nullptr;
    uint32_t *beginCounts = nullptr;   // particles per cell when transport began (per-cell counters on)
    OpacityEos M{};
    Ctx C{};
    // random walk tables (shared by every handle on the device, not owned)
    double *rwTau = nullptr, *rwLogTau = nullptr, *rwSurv = nullptr, *rwRadius = nullptr;
    double *gb = nullptr;            // multigroup bounds
    float *gb32 = nullptr, *gc32 = nullptr;   // multigroup bounds and centres, FP32-tracking form
    double *faceCdf = nullptr;                // multigroup: 6 x (groups + 1) face Planck spectra
    double *mgEp = nullptr, *mgKTq = nullptr; // multigroup: E_g^p per group, (kT)^q per cell
    double4 *ddmc = nullptr;                  // DDMC per-cell data, leak rates, FP32 copy
    double *ddmcTot = nullptr, *ddmcRate = nullptr;
    uint32_t *ddmcCut = nullptr;
    float4 *ddmc32 = nullptr;
    float *ddmcCum32 = nullptr;  // polyhedral FP32 form: cumulative leak fraction per cell-face slot
    double *cfA = nullptr;       // polyhedral mesh: face area per cell-face slot
    // convex-polyhedral mesh
    uint32_t *cfo = nullptr, *cfNext = nullptr, *cfFace = nullptr, *fvo = nullptr, *fvi = nullptr;
    double4 *cfN = nullptr, *cfP = nullptr;
    double *mpx = nullptr, *mpy = nullptr, *mpz = nullptr, *vtx = nullptr, *chord = nullptr;
    float4 *cfN32 = nullptr;
    uint32_t *tetOff = nullptr;  // polyhedral emission: the cells' fan tetrahedra (k_poly_tets)
    double *tetCum = nullptr;
    uint2 *tetAT = nullptr;
    StratParams strat{1, nullptr, 2};         // stratified comb: bins, device bounds, minParticlesPerGroup
    double *stratBounds = nullptr, *stratBinW = nullptr;
    uint32_t *stratStart = nullptr;
    float *mgEp32 = nullptr;
    double faceCdfT[6] = {-1, -1, -1, -1, -1, -1};   // face temperatures the spectra were built for
    // face sources
    uint32_t *fsCell = nullptr;
    int32_t *fsSide = nullptr;
    uint64_t *fsOffset = nullptr;
    uint32_t fsCount = 0;
    uint64_t fsTotal = 0;
    uint32_t *fsFace = nullptr;      // polyhedral meshes: the source faces' indices and areas
    double *fsArea = nullptr;
    // polyhedral meshes: every cell face on the box, in cell and GetCellFaces order
    struct PolyBoundaryFace { uint32_t cell, face; int32_t side; double area; };
    std::vector<PolyBoundaryFace> polyBoundary;
    // banks
    size_t cap = 0;
    Bank bankA{}, bankB{};
    CensusBank bankC{};              // census records (see CensusBank)
    uint64_t *keys = nullptr, *keysAlt = nullptr;
    uint32_t *vals = nullptr, *valsAlt = nullptr, *tileHist = nullptr;
    size_t tileHistLen = 0;
    uint32_t *pCount = nullptr;      // comb: copies per sorted particle
    double *pWeight = nullptr;       // comb: weight of those copies
    uint64_t *pOff = nullptr, *pTiles = nullptr;   // comb: output positions, scan tile sums
    size_t restBytes = 0;            // the block holding bankC.rec through pTiles
    // comb bucket sort scratch, grown on demand: run cursors and scan sums for
    // runLen runs, the list of long runs, and its two flags
    uint32_t *runCursor = nullptr, *longRuns = nullptr, *bucketFlags = nullptr;
    uint64_t *runScan = nullptr;
    size_t runLen = 0, longCap = 0;
    int32_t *dAmbiguous = nullptr;
    // scratch
    uint64_t *offsets = nullptr, *tileSums = nullptr, *dTotalU64 = nullptr;
    double *dTotalE = nullptr, *combW = nullptr, *combWtot = nullptr;
    uint32_t *combStart = nullptr;
    uint64_t *combCount = nullptr;
    uint32_t *counts = nullptr;      // transport round counters (maxRounds + 1) + census counter
    DevStats *dStats = nullptr;
    int32_t *dErr = nullptr;
    // host state
    uint64_t nCensus = 0;            // particles at the head of bankA
    uint64_t nBank = 0;              // particles in bankA after emission
    uint64_t pidLimit = 1;           // every pid of the current census is below this (comb key width)
    // particle shards (storm_cuda_set_sharding): this handle holds shards [shardLo, shardHi) of `shards`
    uint32_t shards = 1, shardLo = 0, shardHi = 1;
    StormExchangeFn exchange = nullptr;
    void *exchangeUser = nullptr;
    std::vector<uint64_t> shardCensus;   // census particles per shard after the last comb (every shard)
    uint64_t nCenGlobal = 0, nCellEmitGlobal = 0, nFaceEmitGlobal = 0;   // this step's global counts
    double *dep = nullptr;           // this handle's material deposits of the step (N)
    double4 *vel = nullptr;          // moving material: (vx, vy, vz, gamma) per cell
    double *egAvg = nullptr;         // group time averages (with_eg_time_avg): ncells x groups
    unsigned long long *fixMat = nullptr, *fixRad = nullptr;   // reproducible tallies: 4 limbs per cell
    double stepDt = 0.0;             // the dt of the step in progress (storm_cuda_phase_begin)
    double *mom = nullptr;           // moving material: momentum, 3 per cell
    double *xbuf = nullptr;          // exchange buffer (max(2 N, 2 S N, S + N) doubles)
    double *shardWc = nullptr;       // cells' global census weights (N)
    double *shardRunW = nullptr;     // run weights (S N)
    uint32_t *shardStart = nullptr;  // run starts (S N + 2)
    uint64_t *shardBounds = nullptr; // 3 (S + 1) pid bounds (Ctx::shardBounds)
    uint32_t step = 0;
    uint32_t K = 8, maxRounds = 4096;
    int minBlocks = 3;               // transport occupancy variant (__launch_bounds__ min blocks); 4 for FP32
    int refill = 1;                  // 1: persistent refill kernel, 0: bank visits of K segments
    uint32_t burst = 8;              // refill kernel: segments between refills
    // online burst tuning (storm_cuda_autotune_transport): step k of the
    // palindromic schedule runs kTuneBursts[order(k)]
    struct {
        uint32_t perCandidate = 0, step = 0;   // perCandidate 0: not tuning
        uint64_t segments[5] = {};
        double ms[5] = {};
    } tune;
    int smCount = 148;
    uint32_t transportGrid = 0;      // resident blocks of the chosen variant x SMs
    uint64_t launches = 0;
    uint64_t exactSums = 0;          // steps whose allocation needed the left-to-right total
    uint64_t memBytes = 0;
    StormStepStats stats{};
    std::vector<uint64_t> lastPhotons;
    double lastTransportMs = 0.0, lastStepMs = 0.0, lastEmitMs = 0.0, lastCombMs = 0.0;
    // transport kernel timing
    bool profiling = false;
    std::vector<cudaEvent_t> evPool;
    double profMs = 0.0;
    uint64_t profLaunches = 0, profSegments = 0;
    int32_t errCode = 0;
    uint64_t errCell = 0, errParticle = 0;
    std::string errMsg;
};

namespace {

int cuda_fail(StormHandle *h, cudaError_t e, const char *what) {
    if (h) {
        h->errMsg = std::string(what) + ": " + cudaGetErrorString(e);
    }
    return e == cudaErrorMemoryAllocation ? STORM_ERR_OOM : STORM_ERR_CUDA;
}

#define CK(call)                                              \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call); \
    } while (0)

// Device memory cache shared by every handle in the process.  cudaFree waits
// for the whole device, so a handle that freed its buffers at the end of a
// request would stall every other problem on the GPU; blocks return here
// instead and are handed to the next allocation of about the same size
// (at most 25% larger) on the same device.  A handle frees only after its own
// stream is idle, so a reused block has no work in flight.
// A miss allocates stream-ordered (cudaMallocFromPoolAsync on the asking
// handle's stream, from the engine's own memory pool on the device, which
// keeps what it maps): plain cudaMalloc, called while other handles' kernels
// ran, was measured to stall for up to hundreds of milliseconds.  The device's
// default pool, which other code in the process may use, is left as it is.
// When the allocation runs out of memory the device's cached blocks are
// released and it retries.
class DevicePool {
public:
    cudaError_t alloc(void **p, size_t bytes, cudaStream_t stream) {
        const size_t want = round_up(bytes);
        int dev = 0;
        cudaGetDevice(&dev);
        {
            std::lock_guard<std::mutex> lk(m_);
            auto it = free_.lower_bound({dev, want});
            if (it != free_.end() && it->first.first == dev && it->first.second <= want + want / 4) {
                *p = it->second;
                live_[it->second] = it->first;
                cached_ -= it->first.second;
                free_.erase(it);
                return cudaSuccess;
            }
        }
        cudaMemPool_t mp = engine_pool(dev);
        cudaError_t e = mp ? cudaMallocFromPoolAsync(p, want, mp, stream) : cudaMalloc(p, want);
        if (e == cudaErrorMemoryAllocation) {
            cudaGetLastError();
            release(dev);
            e = mp ? cudaMallocFromPoolAsync(p, want, mp, stream) : cudaMalloc(p, want);
        }
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> lk(m_);
        live_[*p] = {dev, want};
        ++mallocs_;
        return cudaSuccess;
    }
    void free(void *p) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(m_);
        auto it = live_.find(p);
        if (it == live_.end()) return;
        free_.insert({it->second, p});
        cached_ += it->second.second;
        live_.erase(it);
    }
    // cudaFree every cached block of `dev`; returns the bytes released
    size_t release(int dev) {
        std::vector<void *> blocks;
        size_t bytes = 0;
        {
            std::lock_guard<std::mutex> lk(m_);
            for (auto it = free_.begin(); it != free_.end();) {
                if (it->first.first == dev) {
                    blocks.push_back(it->second);
                    bytes += it->first.second;
                    it = free_.erase(it);
                } else {
                    ++it;
                }
            }
            cached_ -= bytes;
            frees_ += blocks.size();
        }
        int prev = 0;
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
        for (void *b : blocks) cudaFree(b);
        cudaSetDevice(prev);
        return bytes;
    }

    // cudaMalloc and cudaFree calls so far, and the bytes cached and live on all devices
    void counters(uint64_t *mallocs, uint64_t *frees, uint64_t *cached, uint64_t *live) {
        std::lock_guard<std::mutex> lk(m_);
        *mallocs = mallocs_;
        *frees = frees_;
        *cached = cached_;
        uint64_t l = 0;
        for (const auto &kv : live_) l += kv.second.second;
        *live = l;
    }

private:
    // The engine's memory pool on `dev`, created on first use with a release
    // threshold above any size, so it keeps the memory it has mapped (the
    // default threshold, 0, returns memory at every synchronisation); null if
    // the device cannot make one (then plain cudaMalloc).
    cudaMemPool_t engine_pool(int dev) {
        std::lock_guard<std::mutex> lk(m_);
        auto it = pools_.find(dev);
        if (it != pools_.end()) return it->second;
        cudaMemPool_t mp = nullptr;
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        if (cudaMemPoolCreate(&mp, &props) == cudaSuccess) {
            uint64_t threshold = ~0ull;
            cudaMemPoolSetAttribute(mp, cudaMemPoolAttrReleaseThreshold, &threshold);
        } else {
            cudaGetLastError();
            mp = nullptr;
        }
        pools_.emplace(dev, mp);
        return mp;
    }
    static size_t round_up(size_t bytes) {
        if (bytes <= (1u << 20)) {
            size_t b = 512;
            while (b < bytes) b <<= 1;
            return b;
        }
        const size_t g = 2u << 20;
        return (bytes + g - 1) / g * g;
    }
    std::mutex m_;
    std::unordered_map<void *, std::pair<int, size_t>> live_;
    std::multimap<std::pair<int, size_t>, void *> free_;
    size_t cached_ = 0;
    uint64_t mallocs_ = 0, frees_ = 0;
    std::map<int, cudaMemPool_t> pools_;
};

DevicePool &device_pool() {
    static DevicePool pool;
    return pool;
}

// A handle's stream and its six timing events outlive the handle: destroy
// returns them, idle, to a per-device cache and the next create takes them
// from there instead of creating new ones.
constexpr size_t kPinnedBytes = 4096;   // page-locked staging for small readbacks, per stream set
// storm_cuda_step_host: the census upload in at most kHostChunks chunks of at
// least kHostChunkMin particles, each transported once it is in place
constexpr uint32_t kHostChunks = 6;
constexpr uint64_t kHostChunkMin = 1u << 20;
struct StreamSet {
    cudaStream_t stream = nullptr;
    cudaEvent_t ev[6] = {};
    unsigned char *pinned = nullptr;    // kPinnedBytes, or null (readbacks then go to pageable memory)
};
std::mutex &stream_cache_mutex() {
    static std::mutex m;
    return m;
}
std::multimap<int, StreamSet> &stream_cache() {
    static std::multimap<int, StreamSet> c;
    return c;
}
bool take_stream_set(int dev, StreamSet &out) {
    {
        std::lock_guard<std::mutex> lk(stream_cache_mutex());
        auto it = stream_cache().find(dev);
        if (it != stream_cache().end()) {
            out = it->second;
            stream_cache().erase(it);
            return true;
        }
    }
    if (cudaStreamCreateWithFlags(&out.stream, cudaStreamNonBlocking) != cudaSuccess) return false;
    for (cudaEvent_t &e : out.ev)
        if (cudaEventCreate(&e) != cudaSuccess) return false;
    void *p = nullptr;
    if (cudaMallocHost(&p, kPinnedBytes) == cudaSuccess) out.pinned = static_cast<unsigned char *>(p);
    else cudaGetLastError();
    return true;
}
void return_stream_set(int dev, const StreamSet &s) {
    std::lock_guard<std::mutex> lk(stream_cache_mutex());
    stream_cache().emplace(dev, s);
}

template <class T>
cudaError_t dalloc(StormHandle *h, T **p, size_t n) {
    size_t bytes = sizeof(T) * (n ? n : 1);
    cudaError_t e = device_pool().alloc(reinterpret_cast<void **>(p), bytes, h->stream);
    if (e == cudaSuccess) h->memBytes += bytes;
    return e;
}
template <class T>
void dfree(StormHandle *h, T *&p, size_t n) {
    if (p) {
        device_pool().free(p);
        h->memBytes -= sizeof(T) * (n ? n : 1);
        p = nullptr;
    }
}

// A bank's fields live in one device block (one allocation instead of twelve),
// each field on a 256-byte boundary; b.x is the block's start.
size_t align256(size_t bytes) { return (bytes + 255) / 256 * 256; }
size_t bank_bytes(const StormHandle *h, size_t n) {
    const size_t d = align256(n * sizeof(double)), u = align256(n * sizeof(uint32_t));
    return (h->desc.groups >= 2 ? 10 : 9) * d + 3 * u;
}
cudaError_t bank_alloc(StormHandle *h, Bank &b, size_t n) {
    unsigned char *base = nullptr;
    cudaError_t e = dalloc(h, &base, bank_bytes(h, n));
    if (e != cudaSuccess) return e;
    const size_t d = align256(n * sizeof(double)), u = align256(n * sizeof(uint32_t));
    size_t off = 0;
    double **dd[] = {&b.x, &b.y, &b.z, &b.vx, &b.vy, &b.vz, &b.t, &b.w, &b.w0};
    for (double **q : dd) {
        *q = reinterpret_cast<double *>(base + off);
        off += d;
    }
    b.nu = nullptr;
    if (h->desc.groups >= 2) {
        b.nu = reinterpret_cast<double *>(base + off);
        off += d;
    }
    uint32_t **uu[] = {&b.cell, &b.pid, &b.draw};
    for (uint32_t **q : uu) {
        *q = reinterpret_cast<uint32_t *>(base + off);
        off += u;
    }
    return cudaSuccess;
}
void bank_free(StormHandle *h, Bank &b, size_t n) {
    unsigned char *base = reinterpret_cast<unsigned char *>(b.x);
    dfree(h, base, bank_bytes(h, n));
    b = Bank{};
}
cudaError_t bank_copy(cudaStream_t s, const Bank &dst, const Bank &src, size_t n) {
    if (!n) return cudaSuccess;
    const double *sd[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz, src.t, src.w, src.w0};
    double *dd[] = {dst.x, dst.y, dst.z, dst.vx, dst.vy, dst.vz, dst.t, dst.w, dst.w0};
    for (int q = 0; q < 9; ++q) {
        cudaError_t e = cudaMemcpyAsync(dd[q], sd[q], n * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    const uint32_t *su[] = {src.cell, src.pid, src.draw};
    uint32_t *du[] = {dst.cell, dst.pid, dst.draw};
    for (int q = 0; q < 3; ++q) {
        cudaError_t e = cudaMemcpyAsync(du[q], su[q], n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    if (src.nu && dst.nu) {
        cudaError_t e = cudaMemcpyAsync(dst.nu, src.nu, n * sizeof(double), cudaMemcpyDeviceToDevice, s);
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Buffers sized by particle capacity, other than the transport banks A and B.
size_t census_words(const StormHandle *h) { return h->fp32 ? 4 : 6; }   // uint4 per record

// The census records and the comb's sort and plan buffers: one device block,
// each array on a 256-byte boundary, the census records first.
cudaError_t alloc_rest(StormHandle *h, size_t nc) {
    h->tileHistLen = radix_scratch_words(static_cast<uint32_t>(nc));
    void **ptrs[] = {reinterpret_cast<void **>(&h->bankC.rec), reinterpret_cast<void **>(&h->keys),
                     reinterpret_cast<void **>(&h->keysAlt), reinterpret_cast<void **>(&h->vals),
                     reinterpret_cast<void **>(&h->valsAlt), reinterpret_cast<void **>(&h->tileHist),
                     reinterpret_cast<void **>(&h->pCount), reinterpret_cast<void **>(&h->pWeight),
                     reinterpret_cast<void **>(&h->pOff), reinterpret_cast<void **>(&h->pTiles)};
    const size_t bytes[] = {nc * census_words(h) * sizeof(uint4), nc * sizeof(uint64_t), nc * sizeof(uint64_t),
                            nc * sizeof(uint32_t), nc * sizeof(uint32_t), h->tileHistLen * sizeof(*h->tileHist),
                            nc * sizeof(uint32_t), nc * sizeof(double), (nc + 1) * sizeof(uint64_t),
                            (nc / 1024 + 4) * sizeof(uint64_t)};
    size_t total = 0;
    for (size_t b : bytes) total += align256(b);
    unsigned char *base = nullptr;
    cudaError_t e = dalloc(h, &base, total);
    if (e != cudaSuccess) return e;
    h->restBytes = total;
    size_t off = 0;
    for (int q = 0; q < 10; ++q) {
        *ptrs[q] = base + off;
        off += align256(bytes[q]);
    }
    return cudaSuccess;
}
void free_rest(StormHandle *h, size_t) {
    unsigned char *base = reinterpret_cast<unsigned char *>(h->bankC.rec);
    dfree(h, base, h->restBytes);
    h->restBytes = 0;
    h->bankC.rec = nullptr;
    h->keys = h->keysAlt = nullptr;
    h->vals = h->valsAlt = nullptr;
    h->tileHist = nullptr;
    h->pCount = nullptr;
    h->pWeight = nullptr;
    h->pOff = h->pTiles = nullptr;
}

// (Re)allocate every per-particle buffer for capacity n, keeping the first
// `keep` particles of bank A.
int ensure_capacity(StormHandle *h, size_t n, size_t keep) {
    if (n <= h->cap) return STORM_OK;
    if (n > 0xF0000000ull) {
        h->errMsg = "particle count exceeds the 32-bit bank index range";
        return STORM_ERR_CAPACITY;
    }
    size_t nc = std::max<size_t>(n + n / 4, 1u << 16);
    Bank na{};
    CK(bank_alloc(h, na, nc));
    if (keep) CK(bank_copy(h->stream, na, h->bankA, keep));
    CK(cudaStreamSynchronize(h->stream));
    bank_free(h, h->bankA, h->cap);
    bank_free(h, h->bankB, h->cap);
    free_rest(h, h->cap);
    h->bankA = na;
    CK(bank_alloc(h, h->bankB, nc));
    CK(alloc_rest(h, nc));
    h->cap = nc;
    return STORM_OK;
}

// Box-face data from BoundaryCondition::getInwardBoxFaceNormalIfClose
// (boundary/BoundaryCondition.hpp:61-85) evaluated once with the same arithmetic.
void box_faces(StormHandle *h) {
    const double X0 = h->hxe.front(), X1 = h->hxe.back(), Y0 = h->hye.front(), Y1 = h->hye.back(), Z0 = h->hze.front(),
                 Z1 = h->hze.back();
    double V[6][3][3] = {
        {{X0, Y0, Z0}, {X0, Y1, Z0}, {X0, Y1, Z1}}, {{X1, Y0, Z0}, {X1, Y1, Z0}, {X1, Y1, Z1}},
        {{X0, Y0, Z0}, {X0, Y0, Z1}, {X1, Y0, Z1}}, {{X0, Y1, Z0}, {X0, Y1, Z1}, {X1, Y1, Z1}},
        {{X0, Y0, Z0}, {X1, Y0, Z0}, {X1, Y1, Z0}}, {{X0, Y0, Z1}, {X1, Y0, Z1}, {X1, Y1, Z1}},
    };
    const double bc[3] = {0.5 * (X0 + X1), 0.5 * (Y0 + Y1), 0.5 * (Z0 + Z1)};
    for (int f = 0; f < 6; ++f) {
        BoxFaceDev &F = h->C.bf[f];
        double u[3], v[3];
        for (int a = 0; a < 3; ++a) {
            u[a] = V[f][1][a] - V[f][0][a];
            v[a] = V[f][2][a] - V[f][0][a];
            F.on[a] = V[f][0][a];
        }
        F.raw[0] = u[1] * v[2] - u[2] * v[1];
        F.raw[1] = u[2] * v[0] - u[0] * v[2];
        F.raw[2] = u[0] * v[1] - u[1] * v[0];
        double au = std::sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
        double av = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
        double fs = std::min(au, av);
        double nn = std::sqrt(F.raw[0] * F.raw[0] + F.raw[1] * F.raw[1] + F.raw[2] * F.raw[2]);
        F.valid = (nn > 0.0) && std::isfinite(nn) && (fs > 0.0) && std::isfinite(fs);
        F.thresh = 1e-12 * fs * fs * fs;
        F.nudge = 1e-6 * fs;
        h->C.reflNudge[f] = static_cast<float>(F.nudge);
        double inv = 1.0 / nn;
        double n[3] = {F.raw[0] * inv, F.raw[1] * inv, F.raw[2] * inv};
        double tc = n[0] * (bc[0] - F.on[0]) + n[1] * (bc[1] - F.on[1]) + n[2] * (bc[2] - F.on[2]);
        if (tc < 0.0) {
            n[0] *= -1.0; n[1] *= -1.0; n[2] *= -1.0;
        }
        F.unit[0] = n[0]; F.unit[1] = n[1]; F.unit[2] = n[2];
        F.action = h->desc.faces[f].action;
        h->C.sourceT[f] = h->desc.faces[f].source_temperature;
    }
}

// Boundary cell-faces with a source, cells in index order and sides in
// GetCellFaces order (the order generateNewBoundaryParticles visits them).
int build_face_sources(StormHandle *h) {
    std::vector<uint32_t> cell, face;
    std::vector<int32_t> side;
    std::vector<double> area;
    std::vector<uint64_t> off(1, 0);
    const uint32_t nx = h->nx, ny = h->ny, nz = h->nz;
    // a polyhedral mesh: its box faces in cell and GetCellFaces order
    for (const auto &b : h->polyBoundary) {
        const StormBoxFace &bf = h->desc.faces[b.side];
        if (!(bf.source_temperature > 0.0) || bf.packets_per_face == 0) continue;
        cell.push_back(b.cell);
        side.push_back(b.side);
        face.push_back(b.face);
        area.push_back(b.area);
        off.push_back(off.back() + bf.packets_per_face);
    }
    for (uint32_t c = 0; c < (h->C.poly ? 0u : h->N); ++c) {
        uint32_t i = c % nx, j = (c / nx) % ny, k = c / (nx * ny);
        bool bnd[6] = {i == 0, i + 1 == nx, j == 0, j + 1 == ny, k == 0, k + 1 == nz};
        for (int s = 0; s < 6; ++s) {
            if (!bnd[s]) continue;
            const StormBoxFace &bf = h->desc.faces[s];
            if (!(bf.source_temperature > 0.0) || bf.packets_per_face == 0) continue;
            cell.push_back(c);
            side.push_back(s);
            off.push_back(off.back() + bf.packets_per_face);
        }
    }
    dfree(h, h->fsCell, h->fsCount);
    dfree(h, h->fsSide, h->fsCount);
    dfree(h, h->fsOffset, h->fsCount + 1);
    dfree(h, h->fsFace, h->fsCount);
    dfree(h, h->fsArea, h->fsCount);
    h->fsCount = static_cast<uint32_t>(cell.size());
    h->fsTotal = off.back();
    CK(dalloc(h, &h->fsCell, cell.size()));
    CK(dalloc(h, &h->fsSide, side.size()));
    CK(dalloc(h, &h->fsOffset, off.size()));
    CK(dalloc(h, &h->fsFace, cell.size()));
    CK(dalloc(h, &h->fsArea, cell.size()));
    if (!cell.empty()) {
        CK(cudaMemcpyAsync(h->fsCell, cell.data(), cell.size() * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(h->fsSide, side.data(), side.size() * sizeof(int32_t), cudaMemcpyHostToDevice, h->stream));
        if (!face.empty()) {
            CK(cudaMemcpyAsync(h->fsFace, face.data(), face.size() * sizeof(uint32_t), cudaMemcpyHostToDevice,
                               h->stream));
            CK(cudaMemcpyAsync(h->fsArea, area.data(), area.size() * sizeof(double), cudaMemcpyHostToDevice,
                               h->stream));
        }
    }
    CK(cudaMemcpyAsync(h->fsOffset, off.data(), off.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, h->stream));
    // the host vectors go out of scope here
    CK(cudaStreamSynchronize(h->stream));
    return STORM_OK;
}

// RandomWalk tables (radiation/RandomWalk.hpp:23-79): tau and survival on the
// host with the reference's arithmetic, the 1024x256 radius inverse on the device.
double rw_survival(double tau) {
    if (tau <= 0.0 || tau < 1e-4) return 1.0;
    double sum = 0.0;
    const double PI = 3.14159265358979323846;
    for (int n = 1; n <= 500; ++n) {
        double arg = -static_cast<double>(n * n) * PI * PI * tau;
        if (arg < -700.0) break;
        double term = std::exp(arg);
        sum += (n % 2 == 1) ? term : -term;
    }
    double s = 2.0 * sum;
    return s < 0.0 ? 0.0 : (1.0 < s ? 1.0 : s);
}
// The host tables depend on nothing but the table sizes: computed once per process.
struct RwHostTables {
    std::vector<double> tau, ltau, surv;
    RwHostTables() : tau(RW_TABLE), ltau(RW_TABLE), surv(RW_TABLE) {
        const double logMin = std::log(1e-8), logMax = std::log(64.0);
        for (int i = 0; i < RW_TABLE; ++i) {
            double frac = static_cast<double>(i) / static_cast<double>(RW_TABLE - 1);
            tau[i] = std::exp(logMin + frac * (logMax - logMin));
            ltau[i] = std::log(tau[i]);
            surv[i] = rw_survival(tau[i]);
        }
    }
};

// The device tables depend on nothing but constants: built once per device by
// the first handle created there and shared, read-only, by every later handle
// (never freed).  Building them per handle cost a table kernel and a stream
// synchronisation in every storm_cuda_create.
struct RwDeviceTables {
    double *tau = nullptr, *logTau = nullptr, *surv = nullptr, *radius = nullptr;
    float *logTau32 = nullptr, *surv32 = nullptr, *radius32 = nullptr;
    uint16_t *leakStart = nullptr, *leakStart32 = nullptr;
};
// Per bucket b of the survival value, [b, b + 1) / RW_LEAK_BUCKETS: the number
// of table entries above (b + 1) / RW_LEAK_BUCKETS, from which the samplers
// walk forward (the table is non-increasing).  `T` is double for the FP64
// form's table and float for the FP32 copy (the same rounding as the device's).
template <class T>
std::vector<uint16_t> leak_buckets(const std::vector<double> &surv) {
    std::vector<uint16_t> start(RW_LEAK_BUCKETS);
    uint32_t above = 0;
    for (int b = RW_LEAK_BUCKETS - 1; b >= 0; --b) {
        const T top = static_cast<T>(b + 1) / static_cast<T>(RW_LEAK_BUCKETS);
        above = 0;
        while (above < static_cast<uint32_t>(RW_TABLE) && static_cast<T>(surv[above]) > top) ++above;
        start[b] = static_cast<uint16_t>(above);
    }
    return start;
}
std::mutex &rw_tables_mutex() {
    static std::mutex m;
    return m;
}
std::map<int, RwDeviceTables> &rw_tables_by_device() {
    static std::map<int, RwDeviceTables> t;
    return t;
}

int build_rw_tables(StormHandle *h) {
    static const RwHostTables host;   // thread-safe initialisation
    const double logMin = std::log(1e-8), logMax = std::log(64.0);
    std::lock_guard<std::mutex> lk(rw_tables_mutex());
    auto &all = rw_tables_by_device();
    auto it = all.find(h->device);
    if (it == all.end()) {
        RwDeviceTables t;
        const size_t R = static_cast<size_t>(RW_TABLE) * RW_RADIUS;
        CK(cudaMalloc(&t.tau, RW_TABLE * sizeof(double)));
        CK(cudaMalloc(&t.logTau, RW_TABLE * sizeof(double)));
        CK(cudaMalloc(&t.surv, RW_TABLE * sizeof(double)));
        CK(cudaMalloc(&t.radius, R * sizeof(double)));
        CK(cudaMalloc(&t.logTau32, RW_TABLE * sizeof(float)));
        CK(cudaMalloc(&t.surv32, RW_TABLE * sizeof(float)));
        CK(cudaMalloc(&t.radius32, R * sizeof(float)));
        CK(cudaMemcpyAsync(t.tau, host.tau.data(), RW_TABLE * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(t.logTau, host.ltau.data(), RW_TABLE * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(t.surv, host.surv.data(), RW_TABLE * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        {
            static const std::vector<uint16_t> ls = leak_buckets<double>(host.surv), ls32 = leak_buckets<float>(host.surv);
            CK(cudaMalloc(&t.leakStart, RW_LEAK_BUCKETS * sizeof(uint16_t)));
            CK(cudaMalloc(&t.leakStart32, RW_LEAK_BUCKETS * sizeof(uint16_t)));
            CK(cudaMemcpyAsync(t.leakStart, ls.data(), RW_LEAK_BUCKETS * sizeof(uint16_t), cudaMemcpyHostToDevice,
                               h->stream));
            CK(cudaMemcpyAsync(t.leakStart32, ls32.data(), RW_LEAK_BUCKETS * sizeof(uint16_t), cudaMemcpyHostToDevice,
                               h->stream));
        }
        launch_rw_radius(h->stream, t.tau, t.surv, t.radius);
        launch_to_float(h->stream, t.logTau, t.logTau32, RW_TABLE);
        launch_to_float(h->stream, t.surv, t.surv32, RW_TABLE);
        launch_to_float(h->stream, t.radius, t.radius32, RW_TABLE * RW_RADIUS);
        h->launches += 4;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));   // complete before any other handle reads them
        it = all.emplace(h->device, t).first;
    }
    const RwDeviceTables &t = it->second;
    h->rwTau = t.tau;
    h->rwLogTau = t.logTau;
    h->rwSurv = t.surv;
    h->rwRadius = t.radius;
    h->C.rw.tau = t.tau;
    h->C.rw.logTau = t.logTau;
    h->C.rw.surv = t.surv;
    h->C.rw.radius = t.radius;
    h->C.rw.leakStart = t.leakStart;
    if (h->fp32) {
        h->C.rw.logTau32 = t.logTau32;
        h->C.rw.surv32 = t.surv32;
        h->C.rw.radius32 = t.radius32;
        h->C.rw.leakStart32 = t.leakStart32;
    }
    h->C.rw.logMin = logMin;
    h->C.rw.logMax = logMax;
    return STORM_OK;
}

// Small device->host reads on the handle's own stream (never the legacy
// default stream, so handles on other streams keep running), staged through
// the stream set's page-locked buffer: a copy into pageable memory would
// itself wait for the stream, so several reads would drain it several times;
// staged, they complete with one synchronisation.
struct Readback {
    void *dst;
    const void *src;
    size_t bytes;
};
constexpr int kMaxReadbacks = 6;
int raise_from_word(StormHandle *h, const int32_t *e);
// With `check`, the device error word is read as well and a raised error is returned.
int read_many(StormHandle *h, const Readback *r, int n, bool check) {
    int32_t e[3] = {0, 0, 0};
    size_t need = 16;
    for (int q = 0; q < n; ++q) need += (r[q].bytes + 15) / 16 * 16;
    if (h->pinned && n <= kMaxReadbacks && need <= kPinnedBytes) {
        size_t off[kMaxReadbacks + 1];
        size_t o = 0;
        for (int q = 0; q < n; ++q) {
            off[q] = o;
            CK(cudaMemcpyAsync(h->pinned + o, r[q].src, r[q].bytes, cudaMemcpyDeviceToHost, h->stream));
            o += (r[q].bytes + 15) / 16 * 16;
        }
        if (check) CK(cudaMemcpyAsync(h->pinned + o, h->dErr, sizeof(e), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (int q = 0; q < n; ++q) std::memcpy(r[q].dst, h->pinned + off[q], r[q].bytes);
        if (check) std::memcpy(e, h->pinned + o, sizeof(e));
    } else {
        for (int q = 0; q < n; ++q)
            CK(cudaMemcpyAsync(r[q].dst, r[q].src, r[q].bytes, cudaMemcpyDeviceToHost, h->stream));
        if (check) CK(cudaMemcpyAsync(e, h->dErr, sizeof(e), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return check ? raise_from_word(h, e) : STORM_OK;
}

cudaError_t read_small(StormHandle *h, void *dst, const void *src, size_t bytes) {
    if (h->pinned && bytes <= kPinnedBytes) {
        cudaError_t e = cudaMemcpyAsync(h->pinned, src, bytes, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
        if (e == cudaSuccess) std::memcpy(dst, h->pinned, bytes);
        return e;
    }
    cudaError_t e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream);
    if (e != cudaSuccess) return e;
    return cudaStreamSynchronize(h->stream);
}

int check_device_error(StormHandle *h) { return read_many(h, nullptr, 0, true); }

// STORM_ERR_DEVICE with the handle's error fields set when the device error word is raised
int raise_from_word(StormHandle *h, const int32_t *e) {
    if (e[0] != 0) {
        h->errCode = e[0];
        h->errCell = static_cast<uint32_t>(e[1]);
        h->errParticle = static_cast<uint32_t>(e[2]);
        char buf[160];
        std::snprintf(buf, sizeof(buf), "device error %d at cell %u particle %u", e[0], static_cast<uint32_t>(e[1]),
                      static_cast<uint32_t>(e[2]));
        h->errMsg = buf;
        return STORM_ERR_DEVICE;
    }
    return STORM_OK;
}

// One small device->host read together with the device error word, one
// stream synchronisation for both.
int read_checked(StormHandle *h, void *dst, const void *src, size_t bytes) {
    const Readback r{dst, src, bytes};
    return read_many(h, &r, 1, true);
}

void refresh_ctx(StormHandle *h) {
    h->C.step = h->step;
}

// A persistent-style grid: the resident blocks of the variant on every SM (a
// multiple of the SM count), or fewer when the bank is small.
uint32_t grid_transport(uint64_t n, uint32_t resident) {
    uint64_t g = (n + 255) / 256;
    const uint64_t cap = resident ? resident : 148ull * 8;
    if (g < 1) g = 1;
    return static_cast<uint32_t>(g < cap ? g : cap);
}

// refill bursts tried by storm_cuda_autotune_transport, and the candidate of schedule phase p
constexpr uint32_t kTuneBursts[5] = {1, 2, 4, 8, 16};
constexpr uint32_t kTunePhases = 10;   // 1 2 4 8 16 16 8 4 2 1: a linear drift over the steps cancels
uint32_t tune_candidate(uint32_t phase) { return phase < 5 ? phase : 9 - phase; }

}  // namespace

// ====================================================================== C ABI
extern "C" {

int storm_cuda_abi_version(void) { return STORM_CUDA_ABI_VERSION; }

int storm_cuda_release_cached(int device, uint64_t *bytes) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return STORM_ERR_NO_DEVICE;
    if (device < 0 || device >= ndev) return STORM_ERR_INVALID_ARG;
    const size_t b = device_pool().release(device);
    if (bytes) *bytes = b;
    return STORM_OK;
}

int storm_cuda_pool_counters(uint64_t *mallocs, uint64_t *frees, uint64_t *cached_bytes, uint64_t *live_bytes) {
    if (!mallocs || !frees || !cached_bytes || !live_bytes) return STORM_ERR_INVALID_ARG;
    device_pool().counters(mallocs, frees, cached_bytes, live_bytes);
    return STORM_OK;
}

const char *storm_cuda_status_string(int s) {
    switch (s) {
    case STORM_OK: return "ok";
    case STORM_ERR_INVALID_ARG: return "invalid argument";
    case STORM_ERR_CUDA: return "CUDA runtime error";
    case STORM_ERR_OOM: return "device out of memory";
    case STORM_ERR_DEVICE: return "device error word raised";
    case STORM_ERR_CAPACITY: return "particle capacity exceeded";
    case STORM_ERR_UNSUPPORTED: return "unsupported option";
    case STORM_ERR_NO_DEVICE: return "no CUDA device";
    default: return "unknown status";
    }
}

int storm_cuda_create(const StormProblemDesc *d, StormHandle **out) {
    if (!d || !out) return STORM_ERR_INVALID_ARG;
    *out = nullptr;
    if (d->abi_version != STORM_CUDA_ABI_VERSION) return STORM_ERR_INVALID_ARG;
    if (d->nx == 0 || d->ny == 0 || d->nz == 0 || !d->x_edges || !d->y_edges || !d->z_edges) return STORM_ERR_INVALID_ARG;
    if (!d->temperature || !d->mass || !d->internal_energy) return STORM_ERR_INVALID_ARG;
    if (d->new_photons_per_cell == 0) return STORM_ERR_INVALID_ARG;   // RadiationIMC.hpp:584-588
    if ((d->opacity_kind == STORM_OPACITY_CELL_TABLE || d->opacity_kind == STORM_OPACITY_MG_POWER) && !d->sigma_a)
        return STORM_ERR_INVALID_ARG;
    if (d->opacity_kind != STORM_OPACITY_CELL_TABLE && d->opacity_kind != STORM_OPACITY_POWER_LAW &&
        d->opacity_kind != STORM_OPACITY_MG_POWER)
        return STORM_ERR_UNSUPPORTED;
    const bool mg = d->groups >= 2;
    if (mg != (d->opacity_kind == STORM_OPACITY_MG_POWER)) return STORM_ERR_INVALID_ARG;
    if (mg) {   // energyBoundaries must increase (radiation/RadiationIMC.hpp:667-676)
        if (!d->group_bounds || !(d->k_boltz > 0.0) || d->groups > 4096) return STORM_ERR_INVALID_ARG;
        for (uint32_t g = 0; g < d->groups; ++g)
            if (!(d->group_bounds[g + 1] > d->group_bounds[g])) return STORM_ERR_INVALID_ARG;
    }
    if (d->comb_kind != STORM_COMB_PLAIN && d->comb_kind != STORM_COMB_STRATIFIED) return STORM_ERR_INVALID_ARG;
    if (d->comb_kind == STORM_COMB_STRATIFIED) {
        if (d->strat_bins < 1 || d->strat_bins > STORM_STRAT_MAX_BINS) return STORM_ERR_INVALID_ARG;
        if (d->strat_bins > 1 && !d->strat_bounds && !(mg && d->groups == d->strat_bins)) return STORM_ERR_INVALID_ARG;
        const double *sb = d->strat_bounds ? d->strat_bounds : d->group_bounds;
        if (d->strat_bins > 1)
            for (uint32_t g = 0; g < d->strat_bins; ++g)
                if (!(sb[g + 1] > sb[g])) return STORM_ERR_INVALID_ARG;
    }
    if (d->with_ddmc && !(d->ddmc_min_cell_optical_depth >= 0.0 && d->ddmc_min_particle_optical_depth >= 0.0 &&
                          std::isfinite(d->ddmc_min_cell_optical_depth) &&
                          std::isfinite(d->ddmc_min_particle_optical_depth)))
        return STORM_ERR_INVALID_ARG;
    if (d->eos_kind != STORM_EOS_LINEAR && d->eos_kind != STORM_EOS_POWER_LAW) return STORM_ERR_UNSUPPORTED;
    if (d->precision != STORM_PRECISION_FP64 && d->precision != STORM_PRECISION_FP32_TRACK) return STORM_ERR_UNSUPPORTED;
    // moving material: the FP64 form on the Cartesian grid, without DDMC
    if (d->with_hydro && (d->precision != STORM_PRECISION_FP64 || d->mesh || d->with_ddmc)) return STORM_ERR_UNSUPPORTED;
    // reproducible tallies: the transport's deposit and Erad sums only
    if (d->reproducible_tallies && (d->with_hydro || (d->with_eg_time_avg && d->groups >= 2) || !d->comb_enabled))
        return STORM_ERR_UNSUPPORTED;
    if (d->cell_velocity) {
        const uint64_t nv = d->mesh ? d->mesh->ncells : static_cast<uint64_t>(d->nx) * d->ny * d->nz;
        for (uint64_t q = 0; q < 3 * nv; ++q)
            if (!std::isfinite(d->cell_velocity[q]) || !(std::fabs(d->cell_velocity[q]) < d->clight))
                return STORM_ERR_INVALID_ARG;
    }
    const StormPolyMesh *mesh = d->mesh;
    const bool poly = mesh != nullptr;
    uint64_t N64 = poly ? mesh->ncells : static_cast<uint64_t>(d->nx) * d->ny * d->nz;
    if (N64 == 0 || N64 >= 0x7fffffffull) return STORM_ERR_INVALID_ARG;
    if (poly) {
        if (!mesh->points || !mesh->volume || !mesh->cell_face_offset || !mesh->cell_faces || !mesh->face_cells ||
            !mesh->face_normal || !mesh->face_cm || !mesh->face_area || !mesh->face_vertex_offset ||
            !mesh->face_vertices || !mesh->vertices)
            return STORM_ERR_INVALID_ARG;
        if (!(mesh->box[3] > mesh->box[0] && mesh->box[4] > mesh->box[1] && mesh->box[5] > mesh->box[2]))
            return STORM_ERR_INVALID_ARG;
        for (uint32_t c = 0; c < mesh->ncells; ++c)
            if (mesh->cell_face_offset[c + 1] < mesh->cell_face_offset[c]) return STORM_ERR_INVALID_ARG;
        for (uint32_t q = 0; q < mesh->cell_face_offset[mesh->ncells]; ++q)
            if (mesh->cell_faces[q] >= mesh->nfaces) return STORM_ERR_INVALID_ARG;
        for (uint32_t f = 0; f < mesh->nfaces; ++f) {
            if (mesh->face_cells[2 * f] >= mesh->ncells) return STORM_ERR_INVALID_ARG;
            if (mesh->face_vertex_offset[f + 1] < mesh->face_vertex_offset[f]) return STORM_ERR_INVALID_ARG;
        }
        for (uint32_t q = 0; q < mesh->face_vertex_offset[mesh->nfaces]; ++q)
            if (mesh->face_vertices[q] >= mesh->nvertices) return STORM_ERR_INVALID_ARG;
        // the polyhedral kernels are gray: no multigroup opacity
        if (mg) return STORM_ERR_UNSUPPORTED;
    } else {
        for (int a = 0; a < 3; ++a) {
            const double *e = a == 0 ? d->x_edges : (a == 1 ? d->y_edges : d->z_edges);
            uint32_t n = a == 0 ? d->nx : (a == 1 ? d->ny : d->nz);
            for (uint32_t q = 0; q < n; ++q)
                if (!(e[q + 1] > e[q])) return STORM_ERR_INVALID_ARG;
        }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return STORM_ERR_NO_DEVICE;
    if (d->device < 0 || d->device >= ndev) return STORM_ERR_INVALID_ARG;

    StormHandle *h = new StormHandle();
    h->desc = *d;
    h->desc.mesh = nullptr;   // the mesh is copied to the device below; the caller may free it
    h->device = d->device;
    h->nx = poly ? static_cast<uint32_t>(N64) : d->nx;   // a polyhedral mesh: cell_ijk(c) = (c, 0, 0)
    h->ny = poly ? 1 : d->ny;
    h->nz = poly ? 1 : d->nz;
    h->N = static_cast<uint32_t>(N64);
    const uint32_t N = h->N;
    auto fail = [&](int rc) {
        storm_cuda_destroy(h);
        return rc;
    };
    if (cudaSetDevice(h->device) != cudaSuccess) return fail(STORM_ERR_CUDA);
    {
        StreamSet ss;
        const bool ok = take_stream_set(h->device, ss);
        h->stream = ss.stream;
        h->evStart = ss.ev[0]; h->evTransport0 = ss.ev[1]; h->evTransport1 = ss.ev[2];
        h->evEnd = ss.ev[3]; h->evAfterEmit = ss.ev[4]; h->evAfterComb = ss.ev[5];
        h->pinned = ss.pinned;
        if (!ok) return fail(STORM_ERR_CUDA);
    }

    // Cartesian: the edges and centres; a polyhedral mesh: its box as one "cell" per axis
    const uint32_t ex = poly ? 1 : d->nx, ey = poly ? 1 : d->ny, ez = poly ? 1 : d->nz;
    if (poly) {
        h->hxe = {mesh->box[0], mesh->box[3]};
        h->hye = {mesh->box[1], mesh->box[4]};
        h->hze = {mesh->box[2], mesh->box[5]};
    } else {
        h->hxe.assign(d->x_edges, d->x_edges + d->nx + 1);
        h->hye.assign(d->y_edges, d->y_edges + d->ny + 1);
        h->hze.assign(d->z_edges, d->z_edges + d->nz + 1);
    }
    h->hxc.resize(ex); h->hyc.resize(ey); h->hzc.resize(ez);
    for (uint32_t i = 0; i < ex; ++i) h->hxc[i] = 0.5 * (h->hxe[i] + h->hxe[i + 1]);
    for (uint32_t j = 0; j < ey; ++j) h->hyc[j] = 0.5 * (h->hye[j] + h->hye[j + 1]);
    for (uint32_t k = 0; k < ez; ++k) h->hzc[k] = 0.5 * (h->hze[k] + h->hze[k + 1]);

#define ALLOC(ptr, n) do { if (dalloc(h, &(ptr), (n)) != cudaSuccess) return fail(STORM_ERR_OOM); } while (0)
// Every create-time transfer is ordered on the handle's own stream: the legacy
// default stream is not ordered with it (it is created non-blocking).  Pageable
// sources are staged before cudaMemcpyAsync returns; create ends with one
// synchronisation of the stream.
#define H2D(dst, src, n) do { if (cudaMemcpyAsync((dst), (src), sizeof(*(dst)) * (n), cudaMemcpyHostToDevice, h->stream) != cudaSuccess) return fail(STORM_ERR_CUDA); } while (0)
#define ZERO(ptr, bytes) do { if (cudaMemsetAsync((ptr), 0, (bytes), h->stream) != cudaSuccess) return fail(STORM_ERR_CUDA); } while (0)
    ALLOC(h->xe, ex + 1); ALLOC(h->ye, ey + 1); ALLOC(h->ze, ez + 1);
    ALLOC(h->xc, ex); ALLOC(h->yc, ey); ALLOC(h->zc, ez);
    H2D(h->xe, h->hxe.data(), ex + 1); H2D(h->ye, h->hye.data(), ey + 1); H2D(h->ze, h->hze.data(), ez + 1);
    H2D(h->xc, h->hxc.data(), ex); H2D(h->yc, h->hyc.data(), ey); H2D(h->zc, h->hzc.data(), ez);
    h->fp32 = d->precision == STORM_PRECISION_FP32_TRACK;
    // measured on B200 at 64^3: FP32 tracking fits 64 registers without spills (4 blocks of 256
    // per SM); the FP64 form is fastest at 80 registers (3 blocks)
    h->minBlocks = h->fp32 ? 4 : 3;
    if (!poly) {
        std::vector<float> fx(d->nx), fy(d->ny), fz(d->nz);
        for (uint32_t i = 0; i < d->nx; ++i) fx[i] = static_cast<float>(0.5 * (h->hxe[i + 1] - h->hxe[i]));
        for (uint32_t j = 0; j < d->ny; ++j) fy[j] = static_cast<float>(0.5 * (h->hye[j + 1] - h->hye[j]));
        for (uint32_t k = 0; k < d->nz; ++k) fz[k] = static_cast<float>(0.5 * (h->hze[k + 1] - h->hze[k]));
        ALLOC(h->hx, d->nx); ALLOC(h->hy, d->ny); ALLOC(h->hz, d->nz);
        H2D(h->hx, fx.data(), d->nx); H2D(h->hy, fy.data(), d->ny); H2D(h->hz, fz.data(), d->nz);
    }

    CellArrays &A = h->A;
    double **cd[] = {&A.T, &A.mass, &A.vol, &A.eint, &A.ceint, &A.sigA, &A.sigS, &A.fleck, &A.rwSigT, &A.eradAvg,
                     &A.eradCensus, &A.emitE};
    for (double **q : cd) ALLOC(*q, N);
    ALLOC(A.rwElig, N);
    ALLOC(A.photons, N);
    ALLOC(A.phys, N);
    ALLOC(A.phys32, N);
    ALLOC(h->segs, N);
    if (d->per_cell_segment_counters) ALLOC(h->beginCounts, N);
    std::vector<double> vol(N);
    if (poly) {
        vol.assign(mesh->volume, mesh->volume + N);
    } else {
        for (uint32_t c = 0; c < N; ++c) {
            uint32_t i = c % d->nx, j = (c / d->nx) % d->ny, k = c / (d->nx * d->ny);
            vol[c] = (h->hxe[i + 1] - h->hxe[i]) * (h->hye[j + 1] - h->hye[j]) * (h->hze[k + 1] - h->hze[k]);
        }
    }
    H2D(A.vol, vol.data(), N);
    if (poly) {
        // updateGridData (physics/MonteCarloPhysics.hpp:60-84): per cell and face the
        // normal turned toward the cell's mesh point, normalised, and the face centroid
        const uint32_t K = mesh->cell_face_offset[N];
        std::vector<double4> nrm(K), cm(K);
        std::vector<double> area(K);
        std::vector<uint32_t> nextv(K), facev(K);
        std::vector<double> chord(N), mp[3];
        for (int a = 0; a < 3; ++a) mp[a].resize(N);
        for (uint32_t c = 0; c < N; ++c) {
            const double px = mesh->points[3 * c], py = mesh->points[3 * c + 1], pz = mesh->points[3 * c + 2];
            mp[0][c] = px; mp[1][c] = py; mp[2][c] = pz;
            double S = 0.0;
            for (uint32_t q = mesh->cell_face_offset[c]; q < mesh->cell_face_offset[c + 1]; ++q) {
                const uint32_t f = mesh->cell_faces[q];
                double nx = mesh->face_normal[3 * f], ny = mesh->face_normal[3 * f + 1], nz = mesh->face_normal[3 * f + 2];
                const double fx = mesh->face_cm[3 * f], fy = mesh->face_cm[3 * f + 1], fz = mesh->face_cm[3 * f + 2];
                if (nx * (px - fx) + ny * (py - fy) + nz * (pz - fz) < 0) { nx *= -1; ny *= -1; nz *= -1; }
                const double len = std::sqrt(nx * nx + ny * ny + nz * nz);
                if (len > 0) { nx = nx / len; ny = ny / len; nz = nz / len; }
                nrm[q] = make_double4(nx, ny, nz, 0.0);
                cm[q] = make_double4(fx, fy, fz, 0.0);
                area[q] = mesh->face_area[f];
                const uint32_t a0 = mesh->face_cells[2 * f], a1 = mesh->face_cells[2 * f + 1];
                nextv[q] = (a0 == c) ? a1 : a0;
                facev[q] = f;
                S += mesh->face_area[f];   // computeCellSurfaceArea (radiation/RadiationIMC.hpp:971-980)
                if (nextv[q] >= N) {   // a face on the box: its side from the outward normal (-inward),
                                       // as the boundary plug-ins classify it (boundary/SideTemperature.hpp:126-131)
                    const double o[3] = {-nx, -ny, -nz};
                    int side = -1;
                    for (int a = 0; a < 3 && side < 0; ++a) {
                        if (o[a] < -0.99) side = 2 * a;
                        else if (o[a] > 0.99) side = 2 * a + 1;
                    }
                    if (side >= 0) h->polyBoundary.push_back({c, f, side, mesh->face_area[f]});
                }
            }
            chord[c] = (S > 0.0) ? 4.0 * vol[c] / S : 0.0;
        }
        ALLOC(h->cfo, N + 1); ALLOC(h->cfN, K); ALLOC(h->cfP, K); ALLOC(h->cfNext, K); ALLOC(h->cfFace, K);
        ALLOC(h->mpx, N); ALLOC(h->mpy, N); ALLOC(h->mpz, N); ALLOC(h->chord, N);
        const uint32_t NV = mesh->nvertices, FV = mesh->face_vertex_offset[mesh->nfaces];
        ALLOC(h->fvo, mesh->nfaces + 1); ALLOC(h->fvi, FV); ALLOC(h->vtx, 3 * static_cast<size_t>(NV));
        H2D(h->cfo, mesh->cell_face_offset, N + 1);
        H2D(h->cfN, nrm.data(), K); H2D(h->cfP, cm.data(), K); H2D(h->cfNext, nextv.data(), K); H2D(h->cfFace, facev.data(), K);
        ALLOC(h->cfA, K);
        H2D(h->cfA, area.data(), K);
        H2D(h->mpx, mp[0].data(), N); H2D(h->mpy, mp[1].data(), N); H2D(h->mpz, mp[2].data(), N);
        H2D(h->chord, chord.data(), N);
        H2D(h->fvo, mesh->face_vertex_offset, mesh->nfaces + 1);
        H2D(h->fvi, mesh->face_vertices, FV);
        H2D(h->vtx, mesh->vertices, 3 * static_cast<size_t>(NV));
        {   // the emission sampler's tetrahedron table: its offsets here, its sums on the device
            std::vector<uint32_t> toff(static_cast<size_t>(N) + 1);
            uint64_t nt = 0;
            for (uint32_t c = 0; c < N; ++c) {
                toff[c] = static_cast<uint32_t>(nt);
                for (uint32_t q = mesh->cell_face_offset[c]; q < mesh->cell_face_offset[c + 1]; ++q) {
                    const uint32_t nv = mesh->face_vertex_offset[facev[q] + 1] - mesh->face_vertex_offset[facev[q]];
                    if (nv >= 3) nt += nv - 2;
                }
                if (nt > 0xFFFFFFFFull) break;
            }
            if (nt > 0 && nt <= 0xFFFFFFFFull) {   // else the sampler sums the volumes itself
                toff[N] = static_cast<uint32_t>(nt);
                ALLOC(h->tetOff, static_cast<size_t>(N) + 1);
                ALLOC(h->tetCum, nt);
                ALLOC(h->tetAT, nt);
                H2D(h->tetOff, toff.data(), static_cast<size_t>(N) + 1);
            }
        }
        if (d->precision == STORM_PRECISION_FP32_TRACK) {
            // the FP32 form's planes: inward normal and the mesh point's distance from the plane
            std::vector<float4> pl(K);
            for (uint32_t c = 0; c < N; ++c)
                for (uint32_t q = mesh->cell_face_offset[c]; q < mesh->cell_face_offset[c + 1]; ++q) {
                    const double hq = (mp[0][c] - cm[q].x) * nrm[q].x + (mp[1][c] - cm[q].y) * nrm[q].y +
                                      (mp[2][c] - cm[q].z) * nrm[q].z;
                    pl[q] = make_float4(static_cast<float>(nrm[q].x), static_cast<float>(nrm[q].y),
                                        static_cast<float>(nrm[q].z), static_cast<float>(hq));
                }
            ALLOC(h->cfN32, K);
            H2D(h->cfN32, pl.data(), K);
        }
    }
    H2D(A.T, d->temperature, N);
    H2D(A.mass, d->mass, N);
    H2D(A.eint, d->internal_energy, N);
    H2D(A.ceint, d->cell_internal_energy ? d->cell_internal_energy : d->internal_energy, N);
    ZERO(A.eradAvg, N * sizeof(double));
    ZERO(A.eradCensus, N * sizeof(double));
    ZERO(A.sigS, N * sizeof(double));
    ZERO(A.rwElig, N);
    ZERO(A.photons, N * sizeof(uint64_t));
    ZERO(h->segs, N * sizeof(uint32_t));
    if (h->beginCounts) ZERO(h->beginCounts, N * sizeof(uint32_t));
    std::vector<double> ones(N, 1.0);
    H2D(A.fleck, ones.data(), N);

    OpacityEos &M = h->M;
    M.opacityKind = d->opacity_kind;
    M.eosKind = d->eos_kind;
    if (d->opacity_kind == STORM_OPACITY_CELL_TABLE || d->opacity_kind == STORM_OPACITY_MG_POWER) {
        ALLOC(h->tabA, N);
        H2D(h->tabA, d->sigma_a, N);
        // tabS always exists (zeros without sigma_s) so that the per-step
        // opacity refresh (storm_cuda_set_opacity_tables) can fill it
        ALLOC(h->tabS, N);
        if (d->sigma_s) H2D(h->tabS, d->sigma_s, N);
        else ZERO(h->tabS, N * sizeof(double));
    }
    if (d->density_factor) {
        ALLOC(h->rhoF, N);
        H2D(h->rhoF, d->density_factor, N);
    }
    M.tabA = h->tabA; M.tabS = h->tabS; M.rhoF = h->rhoF;
    M.kP0 = d->kP0; M.kR0 = d->kR0; M.alpha = d->alpha; M.tFloor = d->t_floor; M.cap = d->cap;
    M.cvPerMass = d->cv_per_mass; M.eosF = d->eos_f; M.eosBeta = d->eos_beta; M.eosMu = d->eos_mu;

    ALLOC(h->offsets, N + 1);
    ALLOC(h->tileSums, (N + 1023) / 1024 + 1);
    ALLOC(h->dTotalU64, 2);
    ALLOC(h->dTotalE, 2);
    ALLOC(h->combW, N);
    ALLOC(h->combWtot, 2);
    ALLOC(h->combStart, N + 2);
    if (d->comb_kind == STORM_COMB_STRATIFIED) {
        const uint32_t B = d->strat_bins;
        h->strat.bins = B;
        h->strat.minPerBin = d->strat_min_per_bin;
        ALLOC(h->stratStart, static_cast<size_t>(N) * B + 2);
        ALLOC(h->stratBinW, static_cast<size_t>(N) * B);
        if (B > 1) {
            ALLOC(h->stratBounds, B + 1);
            H2D(h->stratBounds, d->strat_bounds ? d->strat_bounds : d->group_bounds, B + 1);
            h->strat.bounds = h->stratBounds;
        }
    }
    ALLOC(h->combCount, N + 1);
    h->maxRounds = d->max_rounds ? d->max_rounds : 16384;
    ALLOC(h->counts, h->maxRounds + 2);
    ALLOC(h->dStats, 1);
    ALLOC(h->dAmbiguous, 2);
    ALLOC(h->dErr, 4);
    ZERO(h->dErr, 4 * sizeof(int32_t));
    h->K = d->segments_per_visit ? d->segments_per_visit : 16;
    // Segments between refills of the persistent transport kernel, measured on
    // B200: multigroup histories are short (about 3.6 segments at 128^3 x 64
    // groups), and lanes idle to the end of a burst once theirs ends, so
    // multigroup problems refill after every segment (against 8: FP32 +23%,
    // FP64 +53% at 2 and a further +28% at 1); polyhedral meshes after 4 (+3%
    // over 8); gray Cartesian grids after 8 (4, 6, 12 and 16 were not faster).
    h->burst = mg ? 1u : (poly ? 4u : 8u);
    {
        // one attribute (cudaGetDeviceProperties queries them all and can take milliseconds)
        int sms = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device) != cudaSuccess || sms <= 0)
            return fail(STORM_ERR_CUDA);
        int nb = transport_blocks_per_sm(h->minBlocks, h->fp32);
        h->transportGrid = static_cast<uint32_t>(sms) * static_cast<uint32_t>(nb > 0 ? nb : 1) * 4;
        h->smCount = sms;
    }

    Ctx &C = h->C;
    C.nx = h->nx; C.ny = h->ny; C.nz = h->nz; C.ncells = N;
    if (poly) {
        C.poly = 1;
        C.cfo = h->cfo; C.cfN = h->cfN; C.cfP = h->cfP; C.cfNext = h->cfNext; C.cfFace = h->cfFace; C.cfA = h->cfA;
        C.mpx = h->mpx; C.mpy = h->mpy; C.mpz = h->mpz;
        C.fvo = h->fvo; C.fvi = h->fvi; C.vtx = h->vtx; C.chord = h->chord; C.cfN32 = h->cfN32;
        if (h->tetCum) {
            launch_poly_tets(h->stream, C, h->tetOff, h->tetCum, h->tetAT);
            if (cudaGetLastError() != cudaSuccess) return fail(STORM_ERR_CUDA);
            C.tetOff = h->tetOff; C.tetCum = h->tetCum; C.tetAT = h->tetAT;
        }
    }
    C.xe = h->xe; C.ye = h->ye; C.ze = h->ze; C.xc = h->xc; C.yc = h->yc; C.zc = h->zc;
    C.X0 = h->hxe.front(); C.X1 = h->hxe.back();
    C.Y0 = h->hye.front(); C.Y1 = h->hye.back();
    C.Z0 = h->hze.front(); C.Z1 = h->hze.back();
    box_faces(h);
    if (mg) {
        const uint32_t G = d->groups;
        ALLOC(h->gb, G + 1);
        H2D(h->gb, d->group_bounds, G + 1);
        ALLOC(A.mgCdf, static_cast<size_t>(N) * (G + 1));
        ALLOC(A.pgrw, N);
        ALLOC(A.pgrwCut, N);
        ALLOC(h->faceCdf, 6 * (static_cast<size_t>(G) + 1));
        ALLOC(h->mgKTq, N);
        {
            // E^p at each group centre with the host's pow, as the opacity
            // model evaluates CalcAbsorptionOpacity there
            std::vector<double> ep(G);
            std::vector<float> ep32(G);
            for (uint32_t g = 0; g < G; ++g) {
                ep[g] = std::pow(0.5 * (d->group_bounds[g] + d->group_bounds[g + 1]), d->mg_p);
                ep32[g] = static_cast<float>(ep[g]);
            }
            ALLOC(h->mgEp, G);
            ALLOC(h->mgEp32, G);
            H2D(h->mgEp, ep.data(), G);
            H2D(h->mgEp32, ep32.data(), G);
        }
        ZERO(A.pgrwCut, N * sizeof(uint32_t));
        C.groups = G;
        C.mgGroupConst = d->mg_group_constant;
        C.gb = h->gb;
        C.mgP = d->mg_p; C.mgQ = d->mg_q; C.mgS = d->mg_s;
        C.kBoltz = d->k_boltz;
        C.sig0 = h->tabA;
        C.mgCdf = A.mgCdf; C.pgrw = A.pgrw; C.pgrwCut = A.pgrwCut;
        C.faceCdf = h->faceCdf;
        C.mgEp = h->mgEp; C.mgEp32 = h->mgEp32; C.mgKTq = h->mgKTq;
        if (h->fp32) {
            std::vector<float> b32(G + 1), c32(G);
            for (uint32_t g = 0; g <= G; ++g) b32[g] = static_cast<float>(d->group_bounds[g]);
            for (uint32_t g = 0; g < G; ++g) c32[g] = static_cast<float>(0.5 * (d->group_bounds[g] + d->group_bounds[g + 1]));
            ALLOC(h->gb32, G + 1);
            ALLOC(h->gc32, G);
            H2D(h->gb32, b32.data(), G + 1);
            H2D(h->gc32, c32.data(), G);
            C.gb32 = h->gb32; C.gc32 = h->gc32;
        }
    }
    C.T = A.T;
    C.escapeNoCheck = d->escape_without_check;
    C.withRW = d->with_random_walk;
    C.noFeedback = d->no_hydro_feedback;
    C.perCellCounters = d->per_cell_segment_counters;
    C.shards = 1;
    C.shardBounds = nullptr;
    // moving material: (vx, vy, vz, gamma) per cell, and the momentum mass * velocity
    C.withHydro = d->with_hydro ? 1 : 0;
    C.invC2 = 1.0 / (d->clight * d->clight);   // units::inv_clight2 = 1 / clight2
    if (d->with_hydro) {
        ALLOC(h->vel, N);
        ALLOC(h->mom, 3 * static_cast<size_t>(N));
        std::vector<double4> v(N);
        std::vector<double> m(3 * static_cast<size_t>(N));
        for (uint32_t c = 0; c < N; ++c) {
            const double vx = d->cell_velocity ? d->cell_velocity[3 * c] : 0.0;
            const double vy = d->cell_velocity ? d->cell_velocity[3 * c + 1] : 0.0;
            const double vz = d->cell_velocity ? d->cell_velocity[3 * c + 2] : 0.0;
            v[c] = make_double4(vx, vy, vz, 1.0);
            m[3 * c] = vx * d->mass[c];
            m[3 * c + 1] = vy * d->mass[c];
            m[3 * c + 2] = vz * d->mass[c];
        }
        H2D(h->vel, v.data(), N);
        H2D(h->mom, m.data(), 3 * static_cast<size_t>(N));
    }
    C.vel = h->vel;
    // group time averages: multigroup problems only (the reference tallies them
    // only with withMultigroupOpacity)
    if (d->with_eg_time_avg && mg) {
        ALLOC(h->egAvg, static_cast<size_t>(N) * d->groups);
        ZERO(h->egAvg, static_cast<size_t>(N) * d->groups * sizeof(double));
    }
    C.egAvg = h->egAvg;
    if (d->reproducible_tallies) {
        ALLOC(h->fixMat, 4 * static_cast<size_t>(N));
        ALLOC(h->fixRad, 4 * static_cast<size_t>(N));
        ZERO(h->fixMat, 4 * static_cast<size_t>(N) * sizeof(unsigned long long));
        ZERO(h->fixRad, 4 * static_cast<size_t>(N) * sizeof(unsigned long long));
    }
    C.fixMat = h->fixMat;
    C.fixRad = h->fixRad;
    C.fixScaleMat = C.fixScaleRad = 1.0;
    C.mom = h->mom;
    C.clight = d->clight; C.arad = d->arad; C.sigmaSB = d->sigma_sb; C.kevKelvin = d->kev_kelvin;
    C.rwMinParticle = d->rw_min_particle_optical_depth;
    C.rwMinCell = d->rw_min_cell_optical_depth;
    if (d->with_ddmc) {
        C.withDDMC = 1;
        C.ddmcPgrw = (d->ddmc_use_multigroup_pgrw && mg) ? 1 : 0;
        C.ddmcMinParticle = d->ddmc_min_particle_optical_depth;
        C.ddmcMinCell = d->ddmc_min_cell_optical_depth;
        ALLOC(h->ddmc, N);
        ALLOC(h->ddmcTot, N);
        // rates per face: 6 per Cartesian cell, one per cell-face slot on a polyhedral mesh
        const size_t rateSlots = poly ? static_cast<size_t>(mesh->cell_face_offset[N]) : 6 * static_cast<size_t>(N);
        ALLOC(h->ddmcRate, rateSlots);
        if (C.ddmcPgrw) ALLOC(h->ddmcCut, N);
        if (h->fp32) ALLOC(h->ddmc32, 3 * static_cast<size_t>(N));
        if (h->fp32 && poly) ALLOC(h->ddmcCum32, rateSlots);
        C.ddmc = h->ddmc; C.ddmcTot = h->ddmcTot; C.ddmcRate = h->ddmcRate; C.ddmcCut = h->ddmcCut;
        C.ddmc32 = h->ddmc32;
        C.ddmcCum32 = h->ddmcCum32;
    }
    C.rwDiffPerReach = C.rwMinParticle > 0.0 ? static_cast<float>(C.clight / (3.0 * C.rwMinParticle)) : 0.0f;
    C.seedLo = static_cast<uint32_t>(d->seed);
    C.seedHi = static_cast<uint32_t>(d->seed >> 32);
    C.step = 0;
    C.phys = A.phys;
    C.phys32 = A.phys32;
    C.fp32 = h->fp32 ? 1 : 0;
    C.hx = h->hx; C.hy = h->hy; C.hz = h->hz;
    C.invC = 1.0 / d->clight;
    C.sigA = A.sigA; C.sigS = A.sigS; C.fleck = A.fleck; C.rwSigT = A.rwSigT; C.rwElig = A.rwElig;
    C.eint = A.eint; C.eradAvg = A.eradAvg; C.segs = h->segs;
    C.err = h->dErr;

    if (build_face_sources(h) != STORM_OK) return fail(STORM_ERR_CUDA);
    if (build_rw_tables(h) != STORM_OK) return fail(STORM_ERR_CUDA);
    size_t cap0 = d->capacity ? d->capacity : std::max<size_t>(1u << 20, N * d->new_photons_per_cell * 4 + h->fsTotal * 2);
    int rc = ensure_capacity(h, cap0, 0);
    if (rc != STORM_OK) return fail(rc);
    // clear the desc's borrowed pointers: the caller may free them after create
    h->desc.x_edges = h->desc.y_edges = h->desc.z_edges = nullptr;
    h->desc.temperature = h->desc.mass = h->desc.internal_energy = h->desc.cell_internal_energy = nullptr;
    h->desc.sigma_a = h->desc.sigma_s = h->desc.density_factor = nullptr;
    if (cudaStreamSynchronize(h->stream) != cudaSuccess) return fail(STORM_ERR_CUDA);
#undef ALLOC
#undef H2D
#undef ZERO
    *out = h;
    return STORM_OK;
}

int storm_cuda_destroy(StormHandle *h) {
    if (!h) return STORM_OK;
    cudaSetDevice(h->device);
    if (h->copyStream) cudaStreamSynchronize(h->copyStream);   // a census upload still writing the banks
    const bool idle = !h->stream || cudaStreamSynchronize(h->stream) == cudaSuccess;
    bank_free(h, h->bankA, h->cap);
    bank_free(h, h->bankB, h->cap);
    free_rest(h, h->cap);
    void *ps[] = {h->xe, h->ye, h->ze, h->xc, h->yc, h->zc, h->A.T, h->A.mass, h->A.vol, h->A.eint, h->A.ceint,
                  h->A.sigA, h->A.sigS, h->A.fleck, h->A.rwSigT, h->A.eradAvg, h->A.eradCensus, h->A.emitE,
                  h->A.rwElig, h->A.photons, h->A.phys, h->A.phys32, h->hx, h->hy, h->hz, h->segs, h->beginCounts, h->tabA, h->tabS, h->rhoF,
                  h->fsCell, h->fsSide, h->fsOffset, h->fsFace, h->fsArea, h->dAmbiguous, h->offsets, h->tileSums, h->dTotalU64, h->dTotalE, h->combW, h->combWtot,
                  h->combStart, h->combCount, h->counts, h->dStats, h->dErr, h->gb, h->A.mgCdf, h->A.pgrw,
                  h->A.pgrwCut, h->gb32, h->gc32, h->faceCdf, h->mgEp, h->mgEp32, h->mgKTq, h->ddmc, h->ddmcTot,
                  h->ddmcRate, h->ddmcCut, h->ddmc32, h->stratBounds, h->stratBinW, h->stratStart,
                  h->runCursor, h->runScan, h->longRuns, h->bucketFlags,
                  h->cfo, h->cfN, h->cfP, h->cfNext, h->cfFace, h->mpx, h->mpy, h->mpz, h->fvo, h->fvi, h->vtx,
                  h->chord, h->cfN32, h->dep, h->xbuf, h->shardWc, h->shardRunW, h->shardStart, h->shardBounds,
                  h->vel, h->mom, h->ddmcCum32, h->cfA, h->egAvg, h->fixMat, h->fixRad, h->tetOff, h->tetCum,
                  h->tetAT};
    for (void *p : ps) device_pool().free(p);
    cudaEvent_t evs[] = {h->evStart, h->evTransport0, h->evTransport1, h->evEnd, h->evAfterEmit, h->evAfterComb};
    bool complete = h->stream != nullptr;
    for (cudaEvent_t e : evs) complete = complete && e;
    if (idle && complete) {
        StreamSet ss;
        ss.stream = h->stream;
        for (int q = 0; q < 6; ++q) ss.ev[q] = evs[q];
        ss.pinned = h->pinned;
        return_stream_set(h->device, ss);
    } else {
        for (cudaEvent_t e : evs)
            if (e) cudaEventDestroy(e);
        if (h->stream) cudaStreamDestroy(h->stream);
        if (h->pinned) cudaFreeHost(h->pinned);
    }
    for (cudaEvent_t e : h->evPool)
        if (e) cudaEventDestroy(e);
    if (h->copyStream) cudaStreamDestroy(h->copyStream);
    for (cudaEvent_t e : {h->evCopyGo, h->evCells})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : h->evChunks)
        if (e) cudaEventDestroy(e);
    delete h;
    return STORM_OK;
}

int storm_cuda_phase_begin(StormHandle *h, double dt) {
    if (!h || !(dt > 0.0)) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    h->errCode = 0;
    h->stepDt = dt;
    h->stats = StormStepStats{};
    CK(cudaMemsetAsync(h->dStats, 0, sizeof(DevStats), h->stream));
    CK(cudaMemsetAsync(h->dErr, 0, 4 * sizeof(int32_t), h->stream));
    refresh_ctx(h);
    h->stats.census_in = h->nCensus;
    // sharded: this handle's census carries the global pids that follow the lower shards' census
    uint64_t pid0 = 0;
    if (h->shards > 1) {
        h->nCenGlobal = 0;
        for (uint32_t q = 0; q < h->shards; ++q) {
            if (q == h->shardLo) pid0 = h->nCenGlobal;
            h->nCenGlobal += h->shardCensus[q];
        }
    } else {
        h->nCenGlobal = h->nCensus;
    }
    if (h->nCensus) {
        launch_begin(h->stream, h->bankA, static_cast<uint32_t>(h->nCensus), static_cast<uint32_t>(pid0), dt,
                     h->dStats);
        ++h->launches;
    }
    h->nBank = h->nCensus;
    CK(cudaGetLastError());
    return STORM_OK;
}

int storm_cuda_phase_prestep(StormHandle *h, double dt) {
    if (!h) return STORM_ERR_INVALID_ARG;
    refresh_ctx(h);
    if (h->egAvg)   // preStep clears Eg_time_avg_ (radiation/RadiationIMC.hpp:1626-1630)
        CK(cudaMemsetAsync(h->egAvg, 0, sizeof(double) * h->N * h->desc.groups, h->stream));
    launch_prestep(h->stream, h->C, h->A, h->M, dt);
    ++h->launches;
    if (h->C.withDDMC) {
        launch_ddmc_rates(h->stream, h->C, h->A);
        ++h->launches;
    }
    CK(cudaGetLastError());
    return STORM_OK;
}

// The emission's first half: the cells' energies and photon counts (the
// reference's allocation, exact) and their scan; *ne gets the step's number of
// cell packets.  Nothing of the handle's state changes but these per-cell counts.
static int emit_count(StormHandle *h, double dt, uint64_t *ne) {
    refresh_ctx(h);
    const uint32_t N = h->N;
    // The reference floors each cell's share against its left-to-right total
    // (RadiationIMC.hpp:2058-2087).  A blocked total plus a rigorous interval
    // settles almost every step; a flagged step recomputes with the exact
    // left-to-right total.  Either way the counts equal the reference's.
    launch_emission_energy(h->stream, h->C, h->A, dt);
    launch_blocked_sum(h->stream, h->A.emitE, N, h->dTotalE);
    CK(cudaMemsetAsync(h->dAmbiguous, 0, sizeof(int32_t), h->stream));
    const double u = 0x1p-53;
    const double rel = 4.0 * (static_cast<double>(N) + 1100.0) * u;   // both orders' rounding, with margin
    launch_allocate_checked(h->stream, h->C, h->A, h->dTotalE, h->desc.new_photons_per_cell, rel, h->dAmbiguous);
    launch_scan_u64(h->stream, h->A.photons, N, h->offsets, h->tileSums, h->dTotalU64);
    h->launches += 6;
    CK(cudaGetLastError());
    struct { uint64_t total; int32_t amb; } back{};
    {
        const Readback r[2] = {{&back.total, h->dTotalU64, sizeof(uint64_t)}, {&back.amb, h->dAmbiguous, sizeof(int32_t)}};
        const int rc = read_many(h, r, 2, false);
        if (rc != STORM_OK) return rc;
    }
    if (back.amb) {
        launch_sequential_sum(h->stream, h->A.emitE, N, h->dTotalE);
        launch_allocate(h->stream, h->C, h->A, h->dTotalE, h->desc.new_photons_per_cell);
        launch_scan_u64(h->stream, h->A.photons, N, h->offsets, h->tileSums, h->dTotalU64);
        h->launches += 5;
        ++h->exactSums;
        CK(cudaGetLastError());
        CK(read_small(h, &back.total, h->dTotalU64, sizeof(uint64_t)));
    }
    *ne = back.total;
    return STORM_OK;
}

// The second half: the material's emission debit and the packets, cell
// packets after the census, face packets after those.
static int emit_packets(StormHandle *h, double dt, uint64_t ne) {
    launch_emission_debit(h->stream, h->C, h->A, h->dStats);
    ++h->launches;
    // The step's packets are numbered over the whole problem: cell packet e has
    // pid nCen + e, face packet f pid nCen + nE + f.  A sharded handle makes
    // its shards' share of each numbering (equal contiguous ranges per shard).
    const uint64_t nf = h->fsTotal;
    h->nCellEmitGlobal = ne;
    h->nFaceEmitGlobal = nf;
    const uint32_t S = h->shards;
    auto cut = [S](uint64_t n, uint32_t sh) {
        return static_cast<uint64_t>((static_cast<unsigned __int128>(n) * sh) / S);
    };
    const uint64_t eLo = cut(ne, h->shardLo), eHi = cut(ne, h->shardHi);
    const uint64_t fLo = cut(nf, h->shardLo), fHi = cut(nf, h->shardHi);
    const uint64_t total = h->nCensus + (eHi - eLo) + (fHi - fLo);
    if (h->nCenGlobal + ne + nf > 0xFFFFFFFFull) return STORM_ERR_CAPACITY;   // pids are 32-bit
    int rc = ensure_capacity(h, total, h->nCensus);
    if (rc != STORM_OK) return rc;
    if (S > 1) {   // the shards' pid bounds: census, cell packets, face packets
        std::vector<uint64_t> bnd(3 * static_cast<size_t>(S + 1));
        uint64_t off = 0;
        for (uint32_t q = 0; q <= S; ++q) {
            bnd[q] = off;
            if (q < S) off += h->shardCensus[q];
            bnd[(S + 1) + q] = h->nCenGlobal + cut(ne, q);
            bnd[2 * (S + 1) + q] = h->nCenGlobal + ne + cut(nf, q);
        }
        CK(cudaMemcpyAsync(h->shardBounds, bnd.data(), bnd.size() * sizeof(uint64_t), cudaMemcpyHostToDevice,
                           h->stream));
        CK(cudaStreamSynchronize(h->stream));   // bnd is pageable and goes out of scope
    }
    launch_emit_cells(h->stream, h->C, h->A, h->offsets, eLo, eHi - eLo, h->bankA, static_cast<uint32_t>(h->nCensus),
                      static_cast<uint32_t>(h->nCenGlobal), dt, h->dStats);
    FaceSources F{h->fsCell, h->fsSide, h->fsOffset, h->fsCount, h->C.poly ? h->fsFace : nullptr,
                  h->C.poly ? h->fsArea : nullptr};
    if (nf && h->C.groups >= 2 && std::memcmp(h->faceCdfT, h->C.sourceT, sizeof(h->faceCdfT)) != 0) {
        launch_face_spectra(h->stream, h->C, h->faceCdf);
        ++h->launches;
        std::memcpy(h->faceCdfT, h->C.sourceT, sizeof(h->faceCdfT));
    }
    launch_emit_faces(h->stream, h->C, F, fLo, fHi - fLo, h->bankA,
                      static_cast<uint32_t>(h->nCensus + (eHi - eLo)), static_cast<uint32_t>(h->nCenGlobal + ne), dt,
                      h->dStats);
    h->launches += (eHi > eLo ? 1 : 0) + (fHi > fLo ? 1 : 0);
    CK(cudaGetLastError());
    h->stats.emitted_cells = eHi - eLo;
    h->stats.emitted_faces = fHi - fLo;
    h->nBank = total;
    return STORM_OK;
}

int storm_cuda_phase_emit(StormHandle *h, double dt) {
    if (!h) return STORM_ERR_INVALID_ARG;
    uint64_t ne = 0;
    const int rc = emit_count(h, dt, &ne);
    return rc != STORM_OK ? rc : emit_packets(h, dt, ne);
}

// Hand `count` doubles of the handle's exchange buffer to the exchange
// callback (an in-place sum over the ranks, ordered on the handle's stream).
static int exchange_sum(StormHandle *h, uint64_t count) {
    if (!h->exchange) return STORM_OK;   // one handle holds every shard
    if (h->exchange(h->exchangeUser, h->xbuf, count, h->stream) != 0) {
        h->errMsg = "the particle-shard exchange callback failed";
        return STORM_ERR_INVALID_ARG;
    }
    return STORM_OK;
}

// Exchange 1 of a sharded step: the per-cell deposits and time-averaged
// radiation tallies summed over the ranks; the deposits then join the
// material energy.
static int exchange_tallies(StormHandle *h) {
    const size_t N = h->N;
    h->C.eint = h->A.eint;
    CK(cudaMemcpyAsync(h->xbuf, h->dep, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    CK(cudaMemcpyAsync(h->xbuf + N, h->A.eradAvg, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    int rc = exchange_sum(h, 2 * N);
    if (rc != STORM_OK) return rc;
    launch_add_into(h->stream, h->A.eint, h->xbuf, static_cast<uint32_t>(N));
    CK(cudaMemcpyAsync(h->A.eradAvg, h->xbuf + N, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    ++h->launches;
    CK(cudaGetLastError());
    return STORM_OK;
}

int storm_cuda_phase_transport(StormHandle *h) {
    if (!h) return STORM_ERR_INVALID_ARG;
    refresh_ctx(h);
    const uint64_t n0 = h->nBank;
    // every pid of the step, over all shards, is below this
    h->pidLimit = h->nCenGlobal + h->nCellEmitGlobal + h->nFaceEmitGlobal;
    if (h->pidLimit == 0) h->pidLimit = 1;
    const bool sharded = h->shards > 1;
    if (sharded) {   // deposits go to a zeroed array first; exchange 1 sums them over the ranks
        CK(cudaMemsetAsync(h->dep, 0, sizeof(double) * h->N, h->stream));
        h->C.eint = h->dep;
    }
    if (h->fixMat) {
        // reproducible tallies: the step's deposits sum to at most the energy of
        // its particles, and its Erad contributions to that energy times dt, so
        // scales that map 4x those bounds below 2^119 keep every partial sum in
        // the limbs, with a unit of 2^-117 of the bound
        DevStats d{};
        CK(read_small(h, &d, h->dStats, sizeof(d)));
        const double E = std::fabs(d.eCensusIn) + std::fabs(d.eEmitted);
        auto scale = [](double bound) {
            if (!(bound > 0.0) || !std::isfinite(bound)) return 1.0;
            int e = 0;
            std::frexp(bound, &e);   // bound < 2^e
            return std::ldexp(1.0, std::min(117 - e, 1000));
        };
        h->C.fixScaleMat = scale(E);
        h->C.fixScaleRad = scale(E * h->stepDt);
        CK(cudaMemsetAsync(h->fixMat, 0, 4 * sizeof(unsigned long long) * h->N, h->stream));
        CK(cudaMemsetAsync(h->fixRad, 0, 4 * sizeof(unsigned long long) * h->N, h->stream));
    }
    CK(cudaEventRecord(h->evTransport0, h->stream));
    CK(cudaMemsetAsync(h->counts, 0, sizeof(uint32_t) * (h->maxRounds + 2), h->stream));
    if (h->desc.per_cell_segment_counters) CK(cudaMemsetAsync(h->segs, 0, sizeof(uint32_t) * h->N, h->stream));
    if (h->beginCounts) {
        CK(cudaMemsetAsync(h->beginCounts, 0, sizeof(uint32_t) * h->N, h->stream));
        launch_cell_histogram(h->stream, h->bankA.cell, static_cast<uint32_t>(n0), h->N, h->beginCounts);
        if (n0) ++h->launches;
    }
    uint32_t n32 = static_cast<uint32_t>(n0);
    uint32_t *nCen = h->counts + h->maxRounds + 1;
    // the multigroup FP32 form runs only in the refill kernel
    const bool refill = h->refill || (h->fp32 && h->desc.groups >= 2) || h->C.poly || h->C.withHydro || h->C.egAvg ||
                        h->C.fixMat;
    if (!refill) CK(cudaMemcpyAsync(h->counts, &n32, sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
    if (refill) {
        // one launch carries every history to census, escape or cutoff
        const uint64_t maxSegs64 = static_cast<uint64_t>(h->maxRounds) * h->K;
        const uint32_t maxSegs = static_cast<uint32_t>(std::min<uint64_t>(maxSegs64, 0xffffffffull));
        int nb = refill_blocks_per_sm(h->minBlocks, h->fp32);
        uint32_t grid = static_cast<uint32_t>(h->smCount) * static_cast<uint32_t>(nb > 0 ? nb : 1);
        const uint32_t need = static_cast<uint32_t>((n0 + 255) / 256);
        if (need < grid) grid = need ? need : 1;
        if (n0) {
            if (h->profiling && h->evPool.empty()) {
                h->evPool.resize(8);
                for (auto &e : h->evPool) CK(cudaEventCreate(&e));
            }
            if (h->profiling) CK(cudaEventRecord(h->evPool[0], h->stream));
            launch_transport_refill(h->stream, grid, h->minBlocks, h->C, h->bankA, n32, h->counts + 1, h->bankC, nCen,
                                    h->burst, maxSegs, h->dStats);
            if (h->profiling) CK(cudaEventRecord(h->evPool[1], h->stream));
            ++h->launches;
        }
        CK(cudaGetLastError());
        CK(cudaEventRecord(h->evTransport1, h->stream));
        uint32_t nc = 0;
        int rc = read_checked(h, &nc, nCen, sizeof(uint32_t));
        if (rc != STORM_OK) return rc;
        if (h->profiling && n0) {
            float ms = 0.f;
            CK(cudaEventElapsedTime(&ms, h->evPool[0], h->evPool[1]));
            h->profMs += ms;
            h->profLaunches += 1;
        }
        h->stats.rounds = n0 ? 1 : 0;
        h->stats.census_out_pre_comb = nc;
        if (h->profiling) {
            DevStats d{};
            CK(read_small(h, &d, h->dStats, sizeof(d)));
            h->profSegments += d.segments;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->evTransport0, h->evTransport1);
        h->lastTransportMs = ms;
        h->nBank = 0;
        return sharded ? exchange_tallies(h) : STORM_OK;
    }
    const uint32_t grid = grid_transport(n0, h->transportGrid);
    uint32_t r = 0;
    bool done = (n0 == 0);
    const uint32_t pollEvery = 4;
    uint32_t remaining = n32;
    if (h->profiling && h->evPool.empty()) {
        h->evPool.resize(2 * pollEvery);
        for (auto &e : h->evPool) CK(cudaEventCreate(&e));
    }
    uint32_t inWindow = 0;
    while (!done && r < h->maxRounds) {
        const Bank &in = (r & 1) ? h->bankB : h->bankA;
        const Bank &out = (r & 1) ? h->bankA : h->bankB;
        if (h->profiling) CK(cudaEventRecord(h->evPool[2 * inWindow], h->stream));
        launch_transport(h->stream, grid, h->C, in, h->counts + r, out, h->counts + r + 1, h->bankC, nCen, h->K,
                         h->dStats, h->minBlocks);
        if (h->profiling) CK(cudaEventRecord(h->evPool[2 * inWindow + 1], h->stream));
        ++inWindow;
        ++h->launches;
        ++r;
        if (r % pollEvery == 0 || r == h->maxRounds) {
            CK(cudaGetLastError());
            CK(cudaMemcpyAsync(&remaining, h->counts + r, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
            CK(cudaStreamSynchronize(h->stream));
            if (h->profiling) {
                for (uint32_t q = 0; q < inWindow; ++q) {
                    float ms = 0.f;
                    CK(cudaEventElapsedTime(&ms, h->evPool[2 * q], h->evPool[2 * q + 1]));
                    h->profMs += ms;
                }
                h->profLaunches += inWindow;
            }
            inWindow = 0;
            if (remaining == 0) done = true;
            int32_t e0 = 0;
            CK(read_small(h, &e0, h->dErr, sizeof(int32_t)));
            if (e0) break;
        }
    }
    CK(cudaEventRecord(h->evTransport1, h->stream));
    h->stats.rounds = r;
    int rc = check_device_error(h);
    if (rc != STORM_OK) return rc;
    if (!done) {
        h->errCode = STORM_DERR_HISTORY_CAP;
        h->errMsg = "transport did not finish within max_rounds bank visits";
        return STORM_ERR_DEVICE;
    }
    uint32_t nc = 0;
    CK(read_small(h, &nc, nCen, sizeof(uint32_t)));
    h->stats.census_out_pre_comb = nc;
    if (h->profiling) {
        DevStats d{};
        CK(read_small(h, &d, h->dStats, sizeof(d)));
        h->profSegments += d.segments;
    }
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->evTransport0, h->evTransport1);
    h->lastTransportMs = ms;
    h->nBank = 0;
    return sharded ? exchange_tallies(h) : STORM_OK;
}

// bits of the comb's pid hash: the smallest b >= 1 with 2^b >= pidLimit
int pid_bits(const StormHandle *h) {
    int b = 1;
    while (b < 32 && (1ull << b) < h->pidLimit) ++b;
    return b;
}

// CombPopulationControl::activate over particle shards (storm_cuda_set_sharding).
// The census is sorted by (shard, cell, keyed hash of pid); the (shard, cell)
// runs' weights and counts go through exchange 2, so that the plan sees every
// cell's global weight and count and each run's offset along its cell; the
// new census stays in (shard, cell) order, and exchange 3 gives every rank the
// shards' census counts and the cells' census energy.  Every rank makes both
// exchanges exactly once per step, whatever its own census holds.
static int comb_sharded(StormHandle *h) {
    const uint32_t n = static_cast<uint32_t>(h->stats.census_out_pre_comb);
    const uint32_t N = h->N, S = h->shards;
    const uint64_t R = static_cast<uint64_t>(S) * N;
    CK(cudaMemsetAsync(h->A.eradCensus, 0, sizeof(double) * N, h->stream));
    const uint32_t combKey = [&] {
        auto fm = [](uint32_t x) {
            x ^= x >> 16; x *= 0x85ebca6bu; x ^= x >> 13; x *= 0xc2b2ae35u; x ^= x >> 16;
            return x;
        };
        return fm(static_cast<uint32_t>(h->desc.seed) ^ fm(h->step * 0x9E3779B9u + static_cast<uint32_t>(h->desc.seed >> 32)));
    }();
    const int pidBits = pid_bits(h);
    int runBits = 0;
    while ((1ull << runBits) <= R) ++runBits;
    if (pidBits + runBits > 64) return STORM_ERR_CAPACITY;
    uint32_t *start = h->shardStart;
    const uint64_t *skeys = h->keysAlt;
    const uint32_t *idx = h->valsAlt;
    double *wS = h->pWeight;
    CombParams P;
    P.nmin = h->desc.comb_nmin;
    P.ntotal = static_cast<uint64_t>(static_cast<double>(static_cast<uint64_t>(N) * h->desc.comb_nmin) * h->desc.comb_factor);
    if (n == 0) {
        CK(cudaMemsetAsync(start, 0, sizeof(uint32_t) * (R + 1), h->stream));
        CK(cudaMemsetAsync(h->dTotalU64, 0, sizeof(uint64_t), h->stream));
    } else {
        launch_comb_keys(h->stream, h->C, h->bankC, n, h->keys, h->vals, combKey, pidBits);
        ++h->launches;
        bool sorted = false;
        if (R + 1 < 0xFFFFFFF0ull) {   // the per-run bucket sort; its flag is read before the exchanges
            const size_t len = R + 1;
            if (len > h->runLen) {
                dfree(h, h->runCursor, h->runLen);
                dfree(h, h->runScan, bucket_scan_words(static_cast<uint32_t>(h->runLen)));
                CK(dalloc(h, &h->runCursor, len));
                CK(dalloc(h, &h->runScan, bucket_scan_words(static_cast<uint32_t>(len))));
                h->runLen = len;
            }
            const size_t longNeed = bucket_long_capacity(n);
            if (longNeed > h->longCap) {
                dfree(h, h->longRuns, h->longCap);
                CK(dalloc(h, &h->longRuns, longNeed));
                h->longCap = longNeed;
            }
            if (!h->bucketFlags) CK(dalloc(h, &h->bucketFlags, 2));
            launch_bucket_sort(h->stream, h->C, h->bankC, h->keys, n, pidBits, static_cast<uint32_t>(R), start,
                               h->runCursor, h->runScan, h->keysAlt, h->valsAlt, wS, h->longRuns,
                               static_cast<uint32_t>(h->longCap), h->bucketFlags);
            h->launches += 7;
            uint32_t flags[2] = {0, 0};
            const Readback r[1] = {{flags, h->bucketFlags, sizeof(flags)}};
            const int rc = read_many(h, r, 1, true);
            if (rc != STORM_OK) return rc;
            sorted = flags[1] == 0;
            if (!sorted) {   // the keys again: the bucket sort consumed them
                launch_comb_keys(h->stream, h->C, h->bankC, n, h->keys, h->vals, combKey, pidBits);
                ++h->launches;
            }
        }
        if (!sorted) {
            const int alt = launch_radix_sort(h->stream, h->keys, h->vals, h->keysAlt, h->valsAlt, n,
                                              pidBits + runBits, h->tileHist);
            skeys = alt ? h->keysAlt : h->keys;
            idx = alt ? h->valsAlt : h->vals;
            launch_comb_ranges(h->stream, skeys, n, static_cast<uint32_t>(R), start, pidBits);
            launch_sorted_weights(h->stream, h->C, h->bankC, idx, n, wS);
            h->launches += 5 * ((pidBits + runBits + 7) / 8) + 2;
        }
    }
    // exchange 2: run weights and counts
    launch_comb_cell_sums(h->stream, wS, start, static_cast<uint32_t>(R), h->shardRunW);
    launch_shard_pack_runs(h->stream, h->shardRunW, start, static_cast<uint32_t>(R), h->xbuf);
    h->launches += 2;
    CK(cudaGetLastError());
    int rc = exchange_sum(h, 2 * R);
    if (rc != STORM_OK) return rc;
    launch_shard_cell_weights(h->stream, h->xbuf, N, S, h->shardWc);
    launch_blocked_sum(h->stream, h->shardWc, N, h->combWtot);
    launch_comb_plan_sharded(h->stream, h->C, P, wS, start, h->xbuf, h->shardWc, h->combWtot, h->shardLo,
                             h->shardHi, h->pCount, h->pWeight, h->A.eradCensus, h->dStats);
    h->launches += 3;
    if (n) {
        uint64_t *countU64 = skeys == h->keysAlt ? h->keys : h->keysAlt;   // the sort's spare key buffer
        launch_mask_count_upto(h->stream, h->pCount, n, start + R, countU64);
        launch_scan_u64(h->stream, countU64, n, h->pOff, h->pTiles, h->dTotalU64);
        h->launches += 4;
    }
    // exchange 3: census particles per shard and census energy per cell
    launch_shard_pack_census(h->stream, h->pOff, h->dTotalU64, start, n, N, S, h->shardLo, h->shardHi,
                             h->A.eradCensus, h->xbuf);
    ++h->launches;
    CK(cudaGetLastError());
    rc = exchange_sum(h, static_cast<uint64_t>(S) + N);
    if (rc != STORM_OK) return rc;
    CK(cudaMemcpyAsync(h->A.eradCensus, h->xbuf + S, N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    std::vector<double> counts(S);
    uint32_t nValid = 0;
    uint64_t total = 0;
    {
        const Readback r[3] = {{counts.data(), h->xbuf, S * sizeof(double)}, {&nValid, start + R, sizeof(uint32_t)},
                               {&total, h->dTotalU64, sizeof(uint64_t)}};
        rc = read_many(h, r, 3, true);
        if (rc != STORM_OK) return rc;
    }
    for (uint32_t q = 0; q < S; ++q) h->shardCensus[q] = static_cast<uint64_t>(counts[q]);
    if (n == 0) nValid = 0;
    size_t grown = 0;
    if (total > h->cap) {
        if (total > 0xF0000000ull) return STORM_ERR_CAPACITY;
        grown = total + total / 4;
        bank_free(h, h->bankA, h->cap);
        bank_free(h, h->bankB, h->cap);
        CK(bank_alloc(h, h->bankA, grown));
        CK(bank_alloc(h, h->bankB, grown));
    }
    if (grown) {
        launch_comb_emit(h->stream, h->C, h->bankC, idx, skeys, pidBits, 1, nValid, h->pCount, h->pWeight, h->pOff,
                         h->bankA);
        ++h->launches;
    } else if (total) {
        uint32_t *src = idx == h->valsAlt ? h->vals : h->valsAlt;   // the sort's spare value buffer
        launch_comb_emit_out(h->stream, h->C, h->bankC, idx, skeys, pidBits, 1, nValid, static_cast<uint32_t>(total),
                             h->pCount, h->pWeight, h->pOff, src, reinterpret_cast<uint32_t *>(h->pTiles), h->bankA);
        h->launches += nValid ? 5 : 0;
    }
    CK(cudaGetLastError());
    if (grown) {
        CK(cudaStreamSynchronize(h->stream));
        free_rest(h, h->cap);
        CK(alloc_rest(h, grown));
        h->cap = grown;
    }
    h->nCensus = total;
    h->stats.census_out = total;
    return STORM_OK;
}

int storm_cuda_phase_comb(StormHandle *h) {
    if (!h) return STORM_ERR_INVALID_ARG;
    refresh_ctx(h);
    if (h->shards > 1) return comb_sharded(h);
    const uint32_t n = static_cast<uint32_t>(h->stats.census_out_pre_comb);
    const uint32_t N = h->N;
    CK(cudaMemsetAsync(h->A.eradCensus, 0, sizeof(double) * N, h->stream));
    if (n == 0) {
        h->nCensus = 0;
        h->stats.census_out = 0;
        return STORM_OK;
    }
    if (!h->desc.comb_enabled) {
        // NoPopulationControl (population/NoPopulationControl.hpp:25-28): the census
        // passes unchanged; order it by pid so the next step's streams are reproducible.
        launch_census_keys_pid(h->stream, h->C, h->bankC, n, h->keys, h->vals);
        int alt = launch_radix_sort(h->stream, h->keys, h->vals, h->keysAlt, h->valsAlt, n, pid_bits(h), h->tileHist);
        const uint32_t *idx = alt ? h->valsAlt : h->vals;
        launch_gather(h->stream, h->C, h->bankC, idx, n, h->bankA, h->A.eradCensus, h->dStats);
        h->launches += 2 + 3 * 4;
        CK(cudaGetLastError());
        h->nCensus = n;
        h->stats.census_out = n;
        return check_device_error(h);
    }
    // CombPopulationControl::activate
    const uint32_t combKey = [&] {
        auto fm = [](uint32_t x) {
            x ^= x >> 16; x *= 0x85ebca6bu; x ^= x >> 13; x *= 0xc2b2ae35u; x ^= x >> 16;
            return x;
        };
        return fm(static_cast<uint32_t>(h->desc.seed) ^ fm(h->step * 0x9E3779B9u + static_cast<uint32_t>(h->desc.seed >> 32)));
    }();
    const int pidBits = pid_bits(h);
    // StratifiedCombPopulationControl sorts by (cell, bin): runs are per (cell, bin)
    const bool strat = h->desc.comb_kind == STORM_COMB_STRATIFIED;
    const uint32_t B = strat ? h->strat.bins : 1u;
    const uint64_t nRuns = static_cast<uint64_t>(N) * B;
    uint32_t *start = strat ? h->stratStart : h->combStart;
    // the key kernel's compact copy of the census weights, for the bucket sort's
    // sorted-weight gather; the plan's output offsets take that space later
    double *wc = reinterpret_cast<double *>(h->pOff);
    if (strat) launch_strat_keys(h->stream, h->C, h->bankC, n, h->keys, h->vals, combKey, pidBits, h->strat, wc);
    else launch_comb_keys(h->stream, h->C, h->bankC, n, h->keys, h->vals, combKey, pidBits, wc);
    int cellBits = 0;
    while ((1ull << cellBits) <= nRuns) ++cellBits;
    // The bucket sort (per-run counting sort, then each run sorted on its own)
    // and the radix sort give the same order; the radix sort is the fallback
    // for runs too long for the bucket sort.  The plan and the scan of the copy
    // counts run on the bucket sort's result before the host learns whether it
    // succeeded: one synchronisation reads the flag, the particle count and the
    // output total together, and only a failed bucket sort repeats the work.
    const uint64_t *skeys = nullptr;
    const uint32_t *idx = nullptr;
    double *wS = h->pWeight;   // census weights in sorted order; the plan overwrites each slot with the copies' weight
    CombParams P;
    P.nmin = h->desc.comb_nmin;
    P.ntotal = static_cast<uint64_t>(static_cast<double>(static_cast<uint64_t>(N) * h->desc.comb_nmin) * h->desc.comb_factor);
    auto radix_sort = [&]() {
        const int alt = launch_radix_sort(h->stream, h->keys, h->vals, h->keysAlt, h->valsAlt, n, pidBits + cellBits,
                                          h->tileHist);
        skeys = alt ? h->keysAlt : h->keys;
        idx = alt ? h->valsAlt : h->vals;
        launch_comb_ranges(h->stream, skeys, n, static_cast<uint32_t>(nRuns), start, pidBits);
        launch_sorted_weights(h->stream, h->C, h->bankC, idx, n, wS);
        h->launches += 5 * ((pidBits + cellBits + 7) / 8) + 2;
    };
    // per-cell sums, the plan, and the copy counts scanned over n slots (the
    // first start[nRuns] are particles, the rest count zero)
    auto plan_and_scan = [&]() {
        if (strat) launch_strat_sums(h->stream, wS, start, N, B, h->stratBinW, h->combW);
        else launch_comb_cell_sums(h->stream, wS, start, N, h->combW);
        launch_blocked_sum(h->stream, h->combW, N, h->combWtot);
        if (strat)
            launch_strat_plan(h->stream, h->C, P, h->strat, wS, start, h->stratBinW, h->combW, h->combWtot, h->pCount,
                              h->pWeight, h->combCount, h->A.eradCensus, h->dStats);
        else
            launch_comb_plan(h->stream, h->C, P, wS, start, h->combW, h->combWtot, h->pCount, h->pWeight,
                             h->combCount, h->A.eradCensus, h->dStats);
        uint64_t *countU64 = skeys == h->keysAlt ? h->keys : h->keysAlt;   // the sort's spare key buffer
        launch_mask_count_upto(h->stream, h->pCount, n, start + nRuns, countU64);
        launch_scan_u64(h->stream, countU64, n, h->pOff, h->pTiles, h->dTotalU64);
        h->launches += 4 + 3;
    };
    bool bucket = false;
    if (nRuns + 1 < 0xFFFFFFF0ull) {
        const size_t len = nRuns + 1;
        if (len > h->runLen) {
            dfree(h, h->runCursor, h->runLen);
            dfree(h, h->runScan, bucket_scan_words(static_cast<uint32_t>(h->runLen)));
            CK(dalloc(h, &h->runCursor, len));
            CK(dalloc(h, &h->runScan, bucket_scan_words(static_cast<uint32_t>(len))));
            h->runLen = len;
        }
        const size_t longNeed = bucket_long_capacity(n);
        if (longNeed > h->longCap) {
            dfree(h, h->longRuns, h->longCap);
            CK(dalloc(h, &h->longRuns, longNeed));
            h->longCap = longNeed;
        }
        if (!h->bucketFlags) CK(dalloc(h, &h->bucketFlags, 2));
        launch_bucket_sort(h->stream, h->C, h->bankC, h->keys, n, pidBits, static_cast<uint32_t>(nRuns), start,
                           h->runCursor, h->runScan, h->keysAlt, h->valsAlt, wS, h->longRuns,
                           static_cast<uint32_t>(h->longCap), h->bucketFlags, wc);
        h->launches += 7;
        skeys = h->keysAlt;
        idx = h->valsAlt;
        bucket = true;
    } else {
        radix_sort();
    }
    plan_and_scan();
    CK(cudaGetLastError());
    uint32_t flags[2] = {0, 0};
    uint32_t nValid = 0;
    uint64_t total = 0;
    {
        const Readback r[3] = {{&nValid, start + nRuns, sizeof(uint32_t)}, {&total, h->dTotalU64, sizeof(uint64_t)},
                               {flags, h->bucketFlags, sizeof(flags)}};
        const int rc = read_many(h, r, bucket ? 3 : 2, true);
        if (rc != STORM_OK) return rc;
    }
    if (bucket && flags[1]) {
        // a run too long for the bucket sort: sort by radix and plan again (the
        // plan adds the census energy to the step statistics, so that restarts)
        CK(cudaMemsetAsync(&h->dStats->eCensusOut, 0, sizeof(double), h->stream));
        // the keys again: the first plan's copy counts went to their buffer
        if (strat) launch_strat_keys(h->stream, h->C, h->bankC, n, h->keys, h->vals, combKey, pidBits, h->strat);
        else launch_comb_keys(h->stream, h->C, h->bankC, n, h->keys, h->vals, combKey, pidBits);
        ++h->launches;
        radix_sort();
        plan_and_scan();
        CK(cudaGetLastError());
        const Readback r[2] = {{&nValid, start + nRuns, sizeof(uint32_t)}, {&total, h->dTotalU64, sizeof(uint64_t)}};
        const int rc = read_many(h, r, 2, true);
        if (rc != STORM_OK) return rc;
    }
    // The write goes to bank A, which transport has finished with.  When the
    // combed census outgrows the banks, A and B are replaced first (their
    // contents are dead); C and the comb buffers, which the write still reads,
    // are replaced after it.
    size_t grown = 0;
    if (total > h->cap) {
        if (total > 0xF0000000ull) return STORM_ERR_CAPACITY;
        grown = total + total / 4;
        bank_free(h, h->bankA, h->cap);
        bank_free(h, h->bankB, h->cap);
        CK(bank_alloc(h, h->bankA, grown));
        CK(bank_alloc(h, h->bankB, grown));
    }
    if (grown) {
        // the output-driven write needs `total` words of scratch, which only the grown buffers have
        launch_comb_emit(h->stream, h->C, h->bankC, idx, skeys, pidBits, B, nValid, h->pCount, h->pWeight, h->pOff,
                         h->bankA);
        ++h->launches;
    } else {
        uint32_t *src = idx == h->valsAlt ? h->vals : h->valsAlt;   // the sort's spare value buffer
        launch_comb_emit_out(h->stream, h->C, h->bankC, idx, skeys, pidBits, B, nValid, static_cast<uint32_t>(total),
                             h->pCount, h->pWeight, h->pOff, src, reinterpret_cast<uint32_t *>(h->pTiles), h->bankA);
        h->launches += nValid && total ? 5 : 0;
    }
    CK(cudaGetLastError());
    if (grown) {
        CK(cudaStreamSynchronize(h->stream));
        free_rest(h, h->cap);
        CK(alloc_rest(h, grown));
        h->cap = grown;
    }
    h->nCensus = total;
    h->stats.census_out = total;
    return STORM_OK;   // errors raised by the comb emit surface at the step's end
}

int poststep_launch(StormHandle *h, double dt) {
    refresh_ctx(h);
    launch_poststep(h->stream, h->C, h->A, h->M, dt);
    ++h->launches;
    CK(cudaGetLastError());
    ++h->step;
    return STORM_OK;
}

int storm_cuda_phase_poststep(StormHandle *h, double dt) {
    if (!h) return STORM_ERR_INVALID_ARG;
    int rc = poststep_launch(h, dt);
    if (rc != STORM_OK) return rc;
    return check_device_error(h);
}

int storm_cuda_phase_stats(StormHandle *h, StormStepStats *s) {
    if (!h || !s) return STORM_ERR_INVALID_ARG;
    DevStats d{};
    CK(read_small(h, &d, h->dStats, sizeof(d)));
    *s = h->stats;
    s->segments = d.segments;
    s->rw_steps = d.rwSteps;
    s->escaped = d.escaped;
    s->cutoff = d.cutoff;
    s->energy_census_in = d.eCensusIn;
    s->energy_emitted = d.eEmitted;
    s->energy_deposited = d.eDeposited;
    s->energy_escaped = d.eEscaped;
    s->energy_census_pre_comb = d.eCensusPre;
    s->energy_census_out = d.eCensusOut;
    s->energy_emission_debit = d.eDebit;
    s->transport_ms = h->lastTransportMs;
    s->step_ms = h->lastStepMs;
    s->emit_ms = h->lastEmitMs;
    s->comb_ms = h->lastCombMs;
    return STORM_OK;
}

int storm_cuda_set_sharding(StormHandle *h, uint32_t shards, uint32_t lo, uint32_t hi, StormExchangeFn exchange,
                            void *user) {
    // once per handle, before its first census
    if (!h || shards == 0 || lo >= hi || hi > shards || h->nCensus != 0 || h->dep) return STORM_ERR_INVALID_ARG;
    if (shards > 1 && (!h->desc.comb_enabled || h->desc.comb_kind != STORM_COMB_PLAIN)) return STORM_ERR_INVALID_ARG;
    if (shards > 1 && (h->C.withHydro || h->C.egAvg || h->C.fixMat))   // tallies without an exchange
        return STORM_ERR_UNSUPPORTED;
    CK(cudaSetDevice(h->device));
    h->shards = shards;
    h->shardLo = lo;
    h->shardHi = hi;
    h->exchange = exchange;
    h->exchangeUser = user;
    h->shardCensus.assign(shards, 0);
    h->C.shards = shards;
    h->C.shardBounds = nullptr;
    if (shards > 1) {
        const size_t N = h->N, R = static_cast<size_t>(shards) * N;
        const size_t xb = std::max({2 * N, 2 * R, static_cast<size_t>(shards) + N});
        CK(dalloc(h, &h->dep, N));
        CK(dalloc(h, &h->xbuf, xb));
        CK(dalloc(h, &h->shardWc, N));
        CK(dalloc(h, &h->shardRunW, R));
        CK(dalloc(h, &h->shardStart, R + 2));
        CK(dalloc(h, &h->shardBounds, 3 * (static_cast<size_t>(shards) + 1)));
        h->C.shardBounds = h->shardBounds;
    }
    return STORM_OK;
}

int storm_cuda_step(StormHandle *h, double dt, StormStepStats *stats) {
    if (!h) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaEventRecord(h->evStart, h->stream));
    int rc = storm_cuda_phase_begin(h, dt);
    if (rc == STORM_OK) rc = storm_cuda_phase_prestep(h, dt);
    if (rc == STORM_OK) rc = storm_cuda_phase_emit(h, dt);
    CK(cudaEventRecord(h->evAfterEmit, h->stream));
    if (rc == STORM_OK) rc = storm_cuda_phase_transport(h);
    if (rc == STORM_OK) rc = storm_cuda_phase_comb(h);
    CK(cudaEventRecord(h->evAfterComb, h->stream));
    if (rc == STORM_OK) rc = poststep_launch(h, dt);
    CK(cudaEventRecord(h->evEnd, h->stream));
    if (rc == STORM_OK) rc = check_device_error(h);   // also waits for the step's last kernel
    CK(cudaEventSynchronize(h->evEnd));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->evStart, h->evEnd);
    h->lastStepMs = ms;
    if (rc == STORM_OK) {
        cudaEventElapsedTime(&ms, h->evStart, h->evAfterEmit);
        h->lastEmitMs = ms;
        cudaEventElapsedTime(&ms, h->evTransport1, h->evAfterComb);
        h->lastCombMs = ms;
    }
    if (rc == STORM_OK && h->tune.perCandidate) {
        // credit this step to the burst it ran with, then move along the schedule
        DevStats d{};
        CK(read_small(h, &d, h->dStats, sizeof(d)));
        const uint32_t c = tune_candidate(h->tune.step / h->tune.perCandidate);
        h->tune.segments[c] += d.segments;
        h->tune.ms[c] += h->lastTransportMs;
        ++h->tune.step;
        if (h->tune.step >= kTunePhases * h->tune.perCandidate) {
            uint32_t best = h->burst;
            double bestRate = -1.0;
            for (uint32_t q = 0; q < 5; ++q) {
                const double rate = h->tune.ms[q] > 0.0 ? static_cast<double>(h->tune.segments[q]) / h->tune.ms[q] : 0.0;
                if (rate > bestRate) {
                    bestRate = rate;
                    best = kTuneBursts[q];
                }
            }
            h->burst = best;
            h->tune = {};
        } else {
            h->burst = kTuneBursts[tune_candidate(h->tune.step / h->tune.perCandidate)];
        }
    }
    if (stats) storm_cuda_phase_stats(h, stats);
    return rc;
}

// storm_cuda_step_host: set_census, step and get_census in one call, the
// census upload overlapped with the step's work that does not need it.  The
// copy stream carries the census into the bank (cells first, checked on the
// device before anything of the step changes the cell state), while the main
// stream runs the prestep, the emission and the transport of the step's new
// packets; the rest of the census follows in chunks, each joining with its
// begin and a transport launch over its slots once it is in place.
// Each particle draws from its own stream and the comb orders the census by
// key, so the result is the three calls' result (FP64 tally sums up to their
// order).  Problems whose transport is not the refill kernel, particle shards,
// moving material, reproducible tallies, the burst tuner and profiling take the
// three calls one after another.
static bool step_host_overlaps(const StormHandle *h) {
    const bool refill = h->refill || (h->fp32 && h->desc.groups >= 2) || h->C.poly || h->C.egAvg;
    return refill && h->shards == 1 && !h->C.withHydro && !h->C.fixMat && !h->tune.perCandidate && !h->profiling &&
           h->pinned != nullptr;
}

static int step_host_overlapped(StormHandle *h, double dt, const StormParticlesSoA *in, StormParticlesSoA *out,
                                uint64_t out_capacity, uint64_t *out_count, StormStepStats *stats) {
    const uint64_t n = in->count;
    const double *sd[] = {in->x, in->y, in->z, in->vx, in->vy, in->vz, in->time_left, in->weight, in->initial_weight};
    if (!in->cell) return STORM_ERR_INVALID_ARG;
    for (int q = 0; q < 9; ++q)
        if (!sd[q] && q != 6 && q != 8) return STORM_ERR_INVALID_ARG;
    if (n > 0xFFFFFFFFull) return STORM_ERR_CAPACITY;
    CK(cudaSetDevice(h->device));
    if (!h->copyStream) {
        CK(cudaStreamCreateWithFlags(&h->copyStream, cudaStreamNonBlocking));
        for (cudaEvent_t *e : {&h->evCopyGo, &h->evCells})
            CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        h->evChunks.assign(kHostChunks, nullptr);
        for (cudaEvent_t &e : h->evChunks) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    // begin (phase_begin without the census's own kernel, which waits for the census)
    h->errCode = 0;
    h->stepDt = dt;
    h->stats = StormStepStats{};
    h->nCensus = 0;
    CK(cudaEventRecord(h->evStart, h->stream));
    CK(cudaMemsetAsync(h->dStats, 0, sizeof(DevStats), h->stream));
    CK(cudaMemsetAsync(h->dErr, 0, 4 * sizeof(int32_t), h->stream));
    refresh_ctx(h);
    int rc = storm_cuda_phase_prestep(h, dt);
    if (rc != STORM_OK) return rc;
    // the step's packet count, then room for census and packets together
    uint64_t ne = 0;
    rc = emit_count(h, dt, &ne);
    if (rc != STORM_OK) return rc;
    if (n + ne + h->fsTotal > 0xFFFFFFFFull) return STORM_ERR_CAPACITY;   // pids are 32-bit
    rc = ensure_capacity(h, n + ne + h->fsTotal, 0);
    if (rc != STORM_OK) return rc;
    // the upload, after every earlier use of the banks on the main stream
    const Bank &stage = h->fp32 ? h->bankB : h->bankA;   // FP32 form: stage FP64, then convert
    double *dd[] = {stage.x, stage.y, stage.z, stage.vx, stage.vy, stage.vz, stage.t, stage.w, stage.w0};
    int32_t *badFlag = reinterpret_cast<int32_t *>(h->pinned + kPinnedBytes - 64);
    cudaStream_t cs = h->copyStream;
    CK(cudaEventRecord(h->evCopyGo, h->stream));
    CK(cudaStreamWaitEvent(cs, h->evCopyGo, 0));
    CK(cudaMemcpyAsync(stage.cell, in->cell, n * sizeof(uint32_t), cudaMemcpyHostToDevice, cs));
    CK(cudaMemsetAsync(h->dAmbiguous + 1, 0, sizeof(int32_t), cs));
    launch_count_bad_cells(cs, stage.cell, static_cast<uint32_t>(n), h->N, h->dAmbiguous + 1);
    ++h->launches;
    CK(cudaMemcpyAsync(badFlag, h->dAmbiguous + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, cs));
    CK(cudaEventRecord(h->evCells, cs));
    // nothing of the cell state changes before the census's cells are known to be in the mesh
    CK(cudaEventSynchronize(h->evCells));
    if (*badFlag) return STORM_ERR_INVALID_ARG;
    // the census's place in the numbering: slots and pids [0, n), packets after it
    h->nCensus = n;
    h->nCenGlobal = n;
    h->stats.census_in = n;
    rc = emit_packets(h, dt, ne);
    if (rc != STORM_OK) return rc;
    CK(cudaEventRecord(h->evAfterEmit, h->stream));
    // transport: the packets [n, nBank), then the census [0, n) once it is in place
    const uint64_t nb = h->nBank;
    h->pidLimit = h->nCenGlobal + h->nCellEmitGlobal + h->nFaceEmitGlobal;   // the comb's key width
    if (h->pidLimit == 0) h->pidLimit = 1;
    CK(cudaEventRecord(h->evTransport0, h->stream));
    CK(cudaMemsetAsync(h->counts, 0, sizeof(uint32_t) * (h->maxRounds + 2), h->stream));
    if (h->desc.per_cell_segment_counters) CK(cudaMemsetAsync(h->segs, 0, sizeof(uint32_t) * h->N, h->stream));
    uint32_t *nCen = h->counts + h->maxRounds + 1;
    const uint64_t maxSegs64 = static_cast<uint64_t>(h->maxRounds) * h->K;
    const uint32_t maxSegs = static_cast<uint32_t>(std::min<uint64_t>(maxSegs64, 0xffffffffull));
    const int nbps = refill_blocks_per_sm(h->minBlocks, h->fp32);
    auto grid_for_range = [&](uint64_t len) {
        uint32_t g = static_cast<uint32_t>(h->smCount) * static_cast<uint32_t>(nbps > 0 ? nbps : 1);
        const uint32_t need = static_cast<uint32_t>((len + 255) / 256);
        return need < g ? (need ? need : 1u) : g;
    };
    if (nb > n) {
        launch_set_u32(h->stream, h->counts + 1, static_cast<uint32_t>(n));   // the refill queue starts at n
        launch_transport_refill(h->stream, grid_for_range(nb - n), h->minBlocks, h->C, h->bankA,
                                static_cast<uint32_t>(nb), h->counts + 1, h->bankC, nCen, h->burst, maxSegs, h->dStats);
        h->launches += 2;
    }
    // the rest of the census behind the work above (from pageable memory the host
    // itself copies while the device runs that work), in chunks that each join
    // the transport as soon as they are in place
    const uint64_t chunk = std::max<uint64_t>(kHostChunkMin, (n + kHostChunks - 1) / kHostChunks);
    uint32_t nChunks = 0;
    for (uint64_t lo = 0; lo < n; lo += chunk, ++nChunks) {
        const uint64_t len = std::min<uint64_t>(chunk, n - lo);
        for (int q = 0; q < 9; ++q) {
            if (sd[q]) CK(cudaMemcpyAsync(dd[q] + lo, sd[q] + lo, len * sizeof(double), cudaMemcpyHostToDevice, cs));
            else CK(cudaMemsetAsync(dd[q] + lo, 0, len * sizeof(double), cs));
        }
        if (stage.nu) {
            if (in->frequency)
                CK(cudaMemcpyAsync(stage.nu + lo, in->frequency + lo, len * sizeof(double), cudaMemcpyHostToDevice, cs));
            else CK(cudaMemsetAsync(stage.nu + lo, 0, len * sizeof(double), cs));
        }
        if (h->fp32) {
            launch_bank_to_local(cs, h->C, h->bankB, h->bankA, static_cast<uint32_t>(lo + len), static_cast<uint32_t>(lo));
            ++h->launches;
        }
        CK(cudaEventRecord(h->evChunks[nChunks], cs));
    }
    CK(cudaGetLastError());
    for (uint32_t k = 0; k < nChunks; ++k) {
        const uint64_t lo = k * chunk, hi = std::min<uint64_t>(n, lo + chunk);
        CK(cudaStreamWaitEvent(h->stream, h->evChunks[k], 0));
        launch_begin(h->stream, h->bankA, static_cast<uint32_t>(hi), 0u, dt, h->dStats, static_cast<uint32_t>(lo));
        ++h->launches;
        if (h->beginCounts && k + 1 == nChunks) {   // every particle's cell is in place now
            CK(cudaMemsetAsync(h->beginCounts, 0, sizeof(uint32_t) * h->N, h->stream));
            launch_cell_histogram(h->stream, h->bankA.cell, static_cast<uint32_t>(nb), h->N, h->beginCounts);
            ++h->launches;
        }
        launch_set_u32(h->stream, h->counts + 1, static_cast<uint32_t>(lo));
        launch_transport_refill(h->stream, grid_for_range(hi - lo), h->minBlocks, h->C, h->bankA,
                                static_cast<uint32_t>(hi), h->counts + 1, h->bankC, nCen, h->burst, maxSegs,
                                h->dStats);
        h->launches += 2;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(h->evTransport1, h->stream));
    uint32_t nc = 0;
    rc = read_checked(h, &nc, nCen, sizeof(uint32_t));
    if (rc != STORM_OK) return rc;
    h->stats.rounds = 1;
    h->stats.census_out_pre_comb = nc;
    float tms = 0.f;
    cudaEventElapsedTime(&tms, h->evTransport0, h->evTransport1);
    h->lastTransportMs = tms;
    h->nBank = 0;
    // the comb, the poststep and the new census back to the host, as storm_cuda_step does
    rc = storm_cuda_phase_comb(h);
    CK(cudaEventRecord(h->evAfterComb, h->stream));
    if (rc == STORM_OK) rc = poststep_launch(h, dt);
    CK(cudaEventRecord(h->evEnd, h->stream));
    if (rc == STORM_OK) rc = check_device_error(h);
    CK(cudaEventSynchronize(h->evEnd));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->evStart, h->evEnd);
    h->lastStepMs = ms;
    if (rc == STORM_OK) {
        cudaEventElapsedTime(&ms, h->evStart, h->evAfterEmit);
        h->lastEmitMs = ms;
        cudaEventElapsedTime(&ms, h->evTransport1, h->evAfterComb);
        h->lastCombMs = ms;
    }
    if (stats) storm_cuda_phase_stats(h, stats);
    if (rc == STORM_OK) rc = storm_cuda_get_census(h, out, out_capacity, out_count);
    return rc;
}

int storm_cuda_step_host(StormHandle *h, double dt, const StormParticlesSoA *in, StormParticlesSoA *out,
                         uint64_t out_capacity, uint64_t *out_count, StormStepStats *stats) {
    if (!h || !in || !out || !(dt > 0.0)) return STORM_ERR_INVALID_ARG;
    if (in->count == 0 || !step_host_overlaps(h)) {
        int rc = storm_cuda_set_census(h, in);
        if (rc == STORM_OK) rc = storm_cuda_step(h, dt, stats);
        if (rc == STORM_OK) rc = storm_cuda_get_census(h, out, out_capacity, out_count);
        return rc;
    }
    const int rc = step_host_overlapped(h, dt, in, out, out_capacity, out_count, stats);
    // a call that failed part-way leaves no upload still writing the banks
    if (rc != STORM_OK && h->copyStream) cudaStreamSynchronize(h->copyStream);
    return rc;
}

// ---------------------------------------------------------------- state in/out
int storm_cuda_set_census(StormHandle *h, const StormParticlesSoA *in) {
    if (!h || !in) return STORM_ERR_INVALID_ARG;
    if (h->shards > 1 && in->count) return STORM_ERR_INVALID_ARG;   // a sharded census is the comb's own
    CK(cudaSetDevice(h->device));
    const uint64_t n = in->count;
    int rc = ensure_capacity(h, n, 0);
    if (rc != STORM_OK) return rc;
    const Bank &stage = h->fp32 ? h->bankB : h->bankA;   // FP32 form: stage FP64, then convert
    const double *sd[] = {in->x, in->y, in->z, in->vx, in->vy, in->vz, in->time_left, in->weight, in->initial_weight};
    double *dd[] = {stage.x, stage.y, stage.z, stage.vx, stage.vy, stage.vz, stage.t, stage.w, stage.w0};
    if (n && !in->cell) return STORM_ERR_INVALID_ARG;
    for (int q = 0; q < 9; ++q)   // time_left (6) and initial_weight (8) may be left out: the step sets them
        if (!sd[q] && n && q != 6 && q != 8) return STORM_ERR_INVALID_ARG;
    h->nCensus = 0;
    if (n) {
        for (int q = 0; q < 9; ++q) {
            if (sd[q]) CK(cudaMemcpyAsync(dd[q], sd[q], n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            else CK(cudaMemsetAsync(dd[q], 0, n * sizeof(double), h->stream));
        }
        CK(cudaMemcpyAsync(stage.cell, in->cell, n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        if (stage.nu) {
            if (in->frequency) CK(cudaMemcpyAsync(stage.nu, in->frequency, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            else CK(cudaMemsetAsync(stage.nu, 0, n * sizeof(double), h->stream));
        }
        // cell indices are checked on the device (a host loop would cost as much as the copy)
        int32_t bad = 0;
        CK(cudaMemsetAsync(h->dAmbiguous + 1, 0, sizeof(int32_t), h->stream));
        launch_count_bad_cells(h->stream, stage.cell, static_cast<uint32_t>(n), h->N, h->dAmbiguous + 1);
        ++h->launches;
        CK(cudaMemcpyAsync(&bad, h->dAmbiguous + 1, sizeof(int32_t), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        if (bad) return STORM_ERR_INVALID_ARG;
        if (h->fp32) {
            launch_bank_to_local(h->stream, h->C, h->bankB, h->bankA, static_cast<uint32_t>(n));
            ++h->launches;
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(h->stream));
        }
    }
    h->nCensus = n;
    return STORM_OK;
}

int storm_cuda_population_control(StormHandle *h, const StormParticlesSoA *in) {
    if (!h || !in) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const uint64_t n = in->count;
    int rc = ensure_capacity(h, n, 0);
    if (rc != STORM_OK) return rc;
    const Bank &stage = h->bankB;   // staged in FP64 layout, then written as census records
    const double *sd[] = {in->x, in->y, in->z, in->vx, in->vy, in->vz, in->time_left, in->weight, in->initial_weight};
    double *dd[] = {stage.x, stage.y, stage.z, stage.vx, stage.vy, stage.vz, stage.t, stage.w, stage.w0};
    if (n) {
        for (int q = 0; q < 9; ++q) {
            if (!sd[q]) return STORM_ERR_INVALID_ARG;
            CK(cudaMemcpyAsync(dd[q], sd[q], n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        }
        if (!in->cell) return STORM_ERR_INVALID_ARG;
        for (uint64_t q = 0; q < n; ++q)
            if (in->cell[q] >= h->N) return STORM_ERR_INVALID_ARG;
        std::vector<uint32_t> pid(n);
        for (uint64_t q = 0; q < n; ++q) pid[q] = static_cast<uint32_t>(q);
        CK(cudaMemcpyAsync(stage.cell, in->cell, n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        CK(cudaMemcpyAsync(stage.pid, pid.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice, h->stream));
        if (stage.nu) {
            if (in->frequency) CK(cudaMemcpyAsync(stage.nu, in->frequency, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
            else CK(cudaMemsetAsync(stage.nu, 0, n * sizeof(double), h->stream));
        }
        CK(cudaMemsetAsync(stage.draw, 0, n * sizeof(uint32_t), h->stream));
        launch_bank_to_census(h->stream, h->C, h->bankB, h->bankC, static_cast<uint32_t>(n));
        ++h->launches;
        CK(cudaGetLastError());
        CK(cudaStreamSynchronize(h->stream));
    }
    CK(cudaMemsetAsync(h->dStats, 0, sizeof(DevStats), h->stream));
    CK(cudaMemsetAsync(h->dErr, 0, 4 * sizeof(int32_t), h->stream));
    h->stats = StormStepStats{};
    h->stats.census_out_pre_comb = n;
    h->pidLimit = n ? n : 1;
    return storm_cuda_phase_comb(h);
}

int storm_cuda_census_count(StormHandle *h, uint64_t *count) {
    if (!h || !count) return STORM_ERR_INVALID_ARG;
    *count = h->nCensus;
    return STORM_OK;
}

int storm_cuda_get_census(StormHandle *h, StormParticlesSoA *out, uint64_t capacity, uint64_t *count) {
    if (!h || !out) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const uint64_t n = std::min<uint64_t>(h->nCensus, capacity);
    if (count) *count = h->nCensus;
    if (h->fp32 && n) {
        launch_bank_to_global(h->stream, h->C, h->bankA, h->bankB, static_cast<uint32_t>(n));
        ++h->launches;
        CK(cudaGetLastError());
    }
    const Bank &src = h->fp32 ? h->bankB : h->bankA;
    const double *sd[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz, src.t, src.w, src.w0};
    double *dd[] = {out->x, out->y, out->z, out->vx, out->vy, out->vz, out->time_left, out->weight, out->initial_weight};
    for (int q = 0; q < 9; ++q)
        if (dd[q] && n) CK(cudaMemcpyAsync(dd[q], sd[q], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (out->cell && n) CK(cudaMemcpyAsync(out->cell, src.cell, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    if (out->frequency && n) {
        if (src.nu) CK(cudaMemcpyAsync(out->frequency, src.nu, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        else std::memset(out->frequency, 0, n * sizeof(double));
    }
    CK(cudaStreamSynchronize(h->stream));
    if (out->id)
        for (uint64_t q = 0; q < n; ++q) out->id[q] = q;
    out->count = n;
    return STORM_OK;
}

int storm_cuda_get_bank(StormHandle *h, StormParticlesSoA *out, uint64_t capacity, uint64_t *count) {
    if (!h) return STORM_ERR_INVALID_ARG;
    if (!out) {   // size query
        if (!count) return STORM_ERR_INVALID_ARG;
        *count = h->nBank;
        return STORM_OK;
    }
    CK(cudaSetDevice(h->device));
    const uint64_t n = std::min<uint64_t>(h->nBank, capacity);
    if (count) *count = h->nBank;
    if (h->fp32 && n) {
        launch_bank_to_global(h->stream, h->C, h->bankA, h->bankB, static_cast<uint32_t>(n));
        ++h->launches;
        CK(cudaGetLastError());
    }
    const Bank &src = h->fp32 ? h->bankB : h->bankA;
    const double *sd[] = {src.x, src.y, src.z, src.vx, src.vy, src.vz, src.t, src.w, src.w0};
    double *dd[] = {out->x, out->y, out->z, out->vx, out->vy, out->vz, out->time_left, out->weight, out->initial_weight};
    for (int q = 0; q < 9; ++q)
        if (dd[q] && n) CK(cudaMemcpyAsync(dd[q], sd[q], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    if (out->cell && n) CK(cudaMemcpyAsync(out->cell, src.cell, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    if (out->frequency && n) {
        if (src.nu) CK(cudaMemcpyAsync(out->frequency, src.nu, n * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        else std::memset(out->frequency, 0, n * sizeof(double));
    }
    std::vector<uint32_t> pid;
    if (out->id && n) {
        pid.resize(n);
        CK(cudaMemcpyAsync(pid.data(), src.pid, n * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    if (out->id)
        for (uint64_t q = 0; q < n; ++q) out->id[q] = pid[q];
    out->count = n;
    return STORM_OK;
}

int storm_cuda_get_cell_arrays(StormHandle *h, double *T, double *eint, double *eradAvg, double *eradCensus,
                               double *sigA, double *fleck, uint64_t *segs) {
    if (!h) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const size_t N = h->N;
    const double *src[] = {h->A.T, h->A.eint, h->A.eradAvg, h->A.eradCensus, h->A.sigA, h->A.fleck};
    double *dst[] = {T, eint, eradAvg, eradCensus, sigA, fleck};
    for (int q = 0; q < 6; ++q)
        if (dst[q]) CK(cudaMemcpyAsync(dst[q], src[q], N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    std::vector<uint32_t> s32;
    if (segs) {
        s32.resize(N);
        CK(cudaMemcpyAsync(s32.data(), h->segs, N * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    }
    CK(cudaStreamSynchronize(h->stream));
    if (segs)
        for (size_t q = 0; q < N; ++q) segs[q] = s32[q];
    return STORM_OK;
}

int storm_cuda_set_cell_state(StormHandle *h, const double *T, const double *eint, const double *ceint) {
    if (!h) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const size_t N = h->N;
    if (T) CK(cudaMemcpyAsync(h->A.T, T, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (eint) CK(cudaMemcpyAsync(h->A.eint, eint, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (ceint) CK(cudaMemcpyAsync(h->A.ceint, ceint, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return STORM_OK;
}

int storm_cuda_set_cell_motion(StormHandle *h, const double *velocity, const double *momentum) {
    if (!h || !h->vel) return STORM_ERR_INVALID_ARG;   // handles created with_hydro only
    CK(cudaSetDevice(h->device));
    const size_t N = h->N;
    if (velocity) {
        std::vector<double4> v(N);
        CK(cudaMemcpyAsync(v.data(), h->vel, N * sizeof(double4), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (size_t c = 0; c < N; ++c) {
            for (int q = 0; q < 3; ++q)
                if (!std::isfinite(velocity[3 * c + q]) || !(std::fabs(velocity[3 * c + q]) < h->C.clight))
                    return STORM_ERR_INVALID_ARG;
            v[c].x = velocity[3 * c]; v[c].y = velocity[3 * c + 1]; v[c].z = velocity[3 * c + 2];
        }
        CK(cudaMemcpyAsync(h->vel, v.data(), N * sizeof(double4), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    if (momentum) {
        CK(cudaMemcpyAsync(h->mom, momentum, 3 * N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return STORM_OK;
}

int storm_cuda_get_group_tallies(StormHandle *h, double *eg_time_avg) {
    if (!h || !eg_time_avg || !h->egAvg) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaMemcpyAsync(eg_time_avg, h->egAvg, sizeof(double) * h->N * h->desc.groups, cudaMemcpyDeviceToHost,
                       h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return STORM_OK;
}

int storm_cuda_get_cell_motion(StormHandle *h, double *velocity, double *momentum) {
    if (!h || !h->vel) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const size_t N = h->N;
    if (velocity) {
        std::vector<double4> v(N);
        CK(cudaMemcpyAsync(v.data(), h->vel, N * sizeof(double4), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
        for (size_t c = 0; c < N; ++c) {
            velocity[3 * c] = v[c].x; velocity[3 * c + 1] = v[c].y; velocity[3 * c + 2] = v[c].z;
        }
    }
    if (momentum) {
        CK(cudaMemcpyAsync(momentum, h->mom, 3 * N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
        CK(cudaStreamSynchronize(h->stream));
    }
    return STORM_OK;
}

int storm_cuda_set_opacity_tables(StormHandle *h, const double *sigA, const double *sigS) {
    if (!h || !h->tabA) return STORM_ERR_INVALID_ARG;   // only the per-cell table opacity kinds have tables
    CK(cudaSetDevice(h->device));
    const size_t N = h->N;
    if (sigA) CK(cudaMemcpyAsync(h->tabA, sigA, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (sigS) CK(cudaMemcpyAsync(h->tabS, sigS, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));   // pageable sources: the caller may reuse them on return
    return STORM_OK;
}

int storm_cuda_get_beginning_counts(StormHandle *h, uint64_t *counts) {
    if (!h || !counts || !h->beginCounts) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    std::vector<uint32_t> c32(h->N);
    CK(cudaMemcpyAsync(c32.data(), h->beginCounts, h->N * sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    for (size_t q = 0; q < h->N; ++q) counts[q] = c32[q];
    return STORM_OK;
}

int storm_cuda_set_cell_physics(StormHandle *h, const double *sigA, const double *sigS, const double *fleck) {
    if (!h) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const size_t N = h->N;
    if (sigA) CK(cudaMemcpyAsync(h->A.sigA, sigA, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (sigS) CK(cudaMemcpyAsync(h->A.sigS, sigS, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (fleck) CK(cudaMemcpyAsync(h->A.fleck, fleck, N * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    launch_rw_eligibility(h->stream, h->C, h->A);
    ++h->launches;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    return STORM_OK;
}

// ---------------------------------------------------------------- checkpoints
// A checkpoint is the state one step hands the next: the census bank as it
// sits on the device (either form's layout, byte for byte), the material state
// of every cell, the face source temperatures and the step counter that keys
// the random streams.  Loaded into a handle created from the same problem, the
// following steps repeat those of the run it was taken from.
namespace {
struct CheckpointHeader {
    char magic[8];               // "STORMCK1"
    uint32_t abi, precision, groups, ncells;
    uint64_t nCensus, step;
    double faceT[6];
};
constexpr size_t kBankArrays = 9;   // x y z vx vy vz t w w0 (8 bytes per particle each)
size_t checkpoint_per_particle(const StormHandle *h) { return kBankArrays * 8 + 3 * 4 + (h->C.groups >= 2 ? 8 : 0); }
size_t checkpoint_bytes(const StormHandle *h, uint64_t n) {
    return sizeof(CheckpointHeader) + n * checkpoint_per_particle(h) + 3 * static_cast<size_t>(h->N) * 8;
}
}  // namespace

int storm_cuda_checkpoint_size(StormHandle *h, uint64_t *bytes) {
    if (!h || !bytes) return STORM_ERR_INVALID_ARG;
    *bytes = checkpoint_bytes(h, h->nCensus);
    return STORM_OK;
}

int storm_cuda_checkpoint_save(StormHandle *h, void *buffer, uint64_t bytes) {
    if (h && h->shards > 1) return STORM_ERR_INVALID_ARG;   // a shard's census is not a problem's
    if (!h || !buffer) return STORM_ERR_INVALID_ARG;
    const uint64_t n = h->nCensus;
    if (bytes < checkpoint_bytes(h, n)) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    char *out = static_cast<char *>(buffer);
    CheckpointHeader hd{};
    std::memcpy(hd.magic, "STORMCK1", 8);
    hd.abi = STORM_CUDA_ABI_VERSION;
    hd.precision = static_cast<uint32_t>(h->desc.precision);
    hd.groups = h->C.groups;
    hd.ncells = h->N;
    hd.nCensus = n;
    hd.step = h->step;
    for (int f = 0; f < 6; ++f) hd.faceT[f] = h->C.sourceT[f];
    std::memcpy(out, &hd, sizeof(hd));
    out += sizeof(hd);
    const Bank &b = h->bankA;
    double *arrs[kBankArrays] = {b.x, b.y, b.z, b.vx, b.vy, b.vz, b.t, b.w, b.w0};
    for (double *a : arrs) {
        if (n) CK(cudaMemcpyAsync(out, a, n * 8, cudaMemcpyDeviceToHost, h->stream));
        out += n * 8;
    }
    uint32_t *ia[3] = {b.cell, b.pid, b.draw};
    for (uint32_t *a : ia) {
        if (n) CK(cudaMemcpyAsync(out, a, n * 4, cudaMemcpyDeviceToHost, h->stream));
        out += n * 4;
    }
    if (h->C.groups >= 2) {
        if (n) CK(cudaMemcpyAsync(out, b.nu, n * 8, cudaMemcpyDeviceToHost, h->stream));
        out += n * 8;
    }
    const double *cells[3] = {h->A.T, h->A.eint, h->A.ceint};
    for (const double *a : cells) {
        CK(cudaMemcpyAsync(out, a, static_cast<size_t>(h->N) * 8, cudaMemcpyDeviceToHost, h->stream));
        out += static_cast<size_t>(h->N) * 8;
    }
    CK(cudaStreamSynchronize(h->stream));
    return STORM_OK;
}

int storm_cuda_checkpoint_load(StormHandle *h, const void *buffer, uint64_t bytes) {
    if (!h || !buffer || bytes < sizeof(CheckpointHeader) || h->shards > 1) return STORM_ERR_INVALID_ARG;
    CheckpointHeader hd;
    std::memcpy(&hd, buffer, sizeof(hd));
    if (std::memcmp(hd.magic, "STORMCK1", 8) != 0 || hd.abi != STORM_CUDA_ABI_VERSION ||
        hd.precision != static_cast<uint32_t>(h->desc.precision) || hd.groups != h->C.groups || hd.ncells != h->N)
        return STORM_ERR_INVALID_ARG;
    // Everything is validated on the host before any of the handle's state is
    // overwritten, so a rejected checkpoint leaves the handle as it was.  The
    // census count comes from the buffer: bound it by the bank's 32-bit indices
    // and by the bytes actually present before sizing anything with it.
    const uint64_t n = hd.nCensus;
    const uint64_t fixedBytes = sizeof(CheckpointHeader) + 3 * static_cast<uint64_t>(h->N) * 8;
    if (bytes < fixedBytes || n > 0xFFFFFFFFull || n > (bytes - fixedBytes) / checkpoint_per_particle(h))
        return STORM_ERR_INVALID_ARG;
    if (bytes < checkpoint_bytes(h, n)) return STORM_ERR_INVALID_ARG;
    for (int f = 0; f < 6; ++f)
        if (!(hd.faceT[f] >= 0.0)) return STORM_ERR_INVALID_ARG;
    {   // the census must name cells of this grid
        const char *cellBytes = static_cast<const char *>(buffer) + sizeof(hd) + kBankArrays * 8 * n;
        for (uint64_t k = 0; k < n; ++k) {
            uint32_t c;
            std::memcpy(&c, cellBytes + 4 * k, sizeof(c));
            if (c >= h->N) return STORM_ERR_INVALID_ARG;
        }
    }
    CK(cudaSetDevice(h->device));
    int rc = ensure_capacity(h, n, 0);
    if (rc != STORM_OK) return rc;
    const char *in = static_cast<const char *>(buffer) + sizeof(hd);
    const Bank &b = h->bankA;
    double *arrs[kBankArrays] = {b.x, b.y, b.z, b.vx, b.vy, b.vz, b.t, b.w, b.w0};
    for (double *a : arrs) {
        if (n) CK(cudaMemcpyAsync(a, in, n * 8, cudaMemcpyHostToDevice, h->stream));
        in += n * 8;
    }
    uint32_t *ia[3] = {b.cell, b.pid, b.draw};
    for (uint32_t *a : ia) {
        if (n) CK(cudaMemcpyAsync(a, in, n * 4, cudaMemcpyHostToDevice, h->stream));
        in += n * 4;
    }
    if (h->C.groups >= 2) {
        if (n) CK(cudaMemcpyAsync(b.nu, in, n * 8, cudaMemcpyHostToDevice, h->stream));
        in += n * 8;
    }
    double *cells[3] = {h->A.T, h->A.eint, h->A.ceint};
    for (double *a : cells) {
        CK(cudaMemcpyAsync(a, in, static_cast<size_t>(h->N) * 8, cudaMemcpyHostToDevice, h->stream));
        in += static_cast<size_t>(h->N) * 8;
    }
    CK(cudaStreamSynchronize(h->stream));
    h->nCensus = n;
    h->step = static_cast<uint32_t>(hd.step);
    for (int f = 0; f < 6; ++f) {
        rc = storm_cuda_set_face_temperature(h, f, hd.faceT[f]);
        if (rc != STORM_OK) return rc;
    }
    return STORM_OK;
}

int storm_cuda_set_face_temperature(StormHandle *h, int face, double T) {
    if (!h || face < 0 || face > 5 || !(T >= 0.0)) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const bool wasSource = h->desc.faces[face].source_temperature > 0.0;
    h->desc.faces[face].source_temperature = T;
    h->C.sourceT[face] = T;
    if (wasSource != (T > 0.0)) return build_face_sources(h);
    return STORM_OK;
}

int storm_cuda_get_emission(StormHandle *h, uint64_t *photons, double *energy) {
    if (!h) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    if (photons) CK(cudaMemcpyAsync(photons, h->A.photons, h->N * sizeof(uint64_t), cudaMemcpyDeviceToHost, h->stream));
    if (energy) CK(cudaMemcpyAsync(energy, h->A.emitE, h->N * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    return STORM_OK;
}

// ---------------------------------------------------------------- parity
int storm_cuda_replay_segments(StormHandle *h, StormReplayBatch *b) {
    if (!h || !b) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    const uint64_t n = b->n;
    if (n == 0) return STORM_OK;
    if (n > 0x7fffffffull) return STORM_ERR_INVALID_ARG;
    uint64_t tapeLen = 0;
    for (uint64_t q = 0; q < n; ++q) tapeLen = std::max<uint64_t>(tapeLen, b->tape_offset[q] + b->tape_length[q]);
    CK(cudaStreamSynchronize(h->stream));
    std::vector<void *> owned;
    auto up = [&](const void *src, size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes ? bytes : 8) != cudaSuccess) return nullptr;
        owned.push_back(p);
        // ordered on the handle's stream, before the replay kernel that reads it
        if (src && bytes) cudaMemcpyAsync(p, src, bytes, cudaMemcpyHostToDevice, h->stream);
        return p;
    };
    ReplayDev R{};
    const double *ins[9] = {b->x, b->y, b->z, b->vx, b->vy, b->vz, b->time_left, b->weight, b->initial_weight};
    for (int q = 0; q < 9; ++q) R.in[q] = static_cast<const double *>(up(ins[q], n * sizeof(double)));
    R.freq = b->frequency ? static_cast<const double *>(up(b->frequency, n * sizeof(double))) : nullptr;
    R.freqOut = b->phys_frequency ? static_cast<double *>(up(nullptr, n * sizeof(double))) : nullptr;
    R.cell = static_cast<const uint32_t *>(up(b->cell, n * sizeof(uint32_t)));
    R.tapeOffset = static_cast<const uint64_t *>(up(b->tape_offset, n * sizeof(uint64_t)));
    R.tapeLength = static_cast<const uint32_t *>(up(b->tape_length, n * sizeof(uint32_t)));
    R.tape = static_cast<const double *>(up(b->tape, tapeLen * sizeof(double)));
    for (int q = 0; q < 8; ++q) R.phys[q] = static_cast<double *>(up(nullptr, n * sizeof(double)));
    for (int q = 0; q < 2; ++q) R.dep[q] = static_cast<double *>(up(nullptr, n * sizeof(double)));
    for (int q = 0; q < 6; ++q) R.mgr[q] = static_cast<double *>(up(nullptr, n * sizeof(double)));
    R.physStatus = static_cast<int32_t *>(up(nullptr, n * sizeof(int32_t)));
    R.physNext = static_cast<uint32_t *>(up(nullptr, n * sizeof(uint32_t)));
    R.mgrCell = static_cast<uint32_t *>(up(nullptr, n * sizeof(uint32_t)));
    R.mgrStatus = static_cast<int32_t *>(up(nullptr, n * sizeof(int32_t)));
    R.draws = static_cast<uint32_t *>(up(nullptr, n * sizeof(uint32_t)));
    R.usedRW = static_cast<int32_t *>(up(nullptr, n * sizeof(int32_t)));
    R.momOut = b->phys_momentum ? static_cast<double *>(up(nullptr, 3 * n * sizeof(double))) : nullptr;
    bool ok = true;
    for (void *p : owned) ok = ok && p;
    int rc = STORM_OK;
    if (!ok) rc = STORM_ERR_OOM;
    if (rc == STORM_OK) {
        refresh_ctx(h);
        launch_replay(h->stream, h->C, R, static_cast<uint32_t>(n));
        ++h->launches;
        if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(h->stream) != cudaSuccess) rc = STORM_ERR_CUDA;
    }
    if (rc == STORM_OK) {
        double *ph[8] = {b->phys_x, b->phys_y, b->phys_z, b->phys_vx, b->phys_vy, b->phys_vz, b->phys_time_left,
                         b->phys_weight};
        for (int q = 0; q < 8; ++q) cudaMemcpy(ph[q], R.phys[q], n * sizeof(double), cudaMemcpyDeviceToHost);
        double *mg[6] = {b->mgr_x, b->mgr_y, b->mgr_z, b->mgr_vx, b->mgr_vy, b->mgr_vz};
        for (int q = 0; q < 6; ++q) cudaMemcpy(mg[q], R.mgr[q], n * sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->dep_material, R.dep[0], n * sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->dep_erad, R.dep[1], n * sizeof(double), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->phys_status, R.physStatus, n * sizeof(int32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->phys_next_cell, R.physNext, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->mgr_cell, R.mgrCell, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->mgr_status, R.mgrStatus, n * sizeof(int32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->draws_used, R.draws, n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
        cudaMemcpy(b->used_random_walk, R.usedRW, n * sizeof(int32_t), cudaMemcpyDeviceToHost);
        if (b->phys_frequency) cudaMemcpy(b->phys_frequency, R.freqOut, n * sizeof(double), cudaMemcpyDeviceToHost);
        if (b->phys_momentum) cudaMemcpy(b->phys_momentum, R.momOut, 3 * n * sizeof(double), cudaMemcpyDeviceToHost);
    }
    for (void *p : owned)
        if (p) cudaFree(p);
    return rc;
}

int storm_cuda_get_random_walk_tables(StormHandle *h, double *tau, double *survival, double *radius) {
    if (!h) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    if (tau) CK(cudaMemcpy(tau, h->rwTau, RW_TABLE * sizeof(double), cudaMemcpyDeviceToHost));
    if (survival) CK(cudaMemcpy(survival, h->rwSurv, RW_TABLE * sizeof(double), cudaMemcpyDeviceToHost));
    if (radius)
        CK(cudaMemcpy(radius, h->rwRadius, static_cast<size_t>(RW_TABLE) * RW_RADIUS * sizeof(double),
                      cudaMemcpyDeviceToHost));
    return STORM_OK;
}

int storm_cuda_random_walk_sample(StormHandle *h, uint64_t n, const double *xiLeak, const double *tau,
                                  const double *xiRad, double *leakOut, double *radOut) {
    if (!h || n == 0 || n > 0x7fffffffull) return STORM_ERR_INVALID_ARG;
    CK(cudaSetDevice(h->device));
    CK(cudaStreamSynchronize(h->stream));
    double *d[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    for (int q = 0; q < 5; ++q) CK(cudaMalloc(&d[q], n * sizeof(double)));
    if (xiLeak) CK(cudaMemcpyAsync(d[0], xiLeak, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (tau) CK(cudaMemcpyAsync(d[1], tau, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    if (xiRad) CK(cudaMemcpyAsync(d[2], xiRad, n * sizeof(double), cudaMemcpyHostToDevice, h->stream));
    launch_rw_sample(h->stream, h->C.rw, static_cast<uint32_t>(n), xiLeak ? d[0] : nullptr, tau ? d[1] : nullptr,
                     xiRad ? d[2] : nullptr, d[3], d[4]);
    ++h->launches;
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    if (leakOut && xiLeak) CK(cudaMemcpy(leakOut, d[3], n * sizeof(double), cudaMemcpyDeviceToHost));
    if (radOut && tau && xiRad) CK(cudaMemcpy(radOut, d[4], n * sizeof(double), cudaMemcpyDeviceToHost));
    for (int q = 0; q < 5; ++q) cudaFree(d[q]);
    return STORM_OK;
}

// ---------------------------------------------------------------- diagnostics
int storm_cuda_last_error(StormHandle *h, int32_t *derr, uint64_t *cell, uint64_t *particle, char *msg, size_t len) {
    if (!h) return STORM_ERR_INVALID_ARG;
    if (derr) *derr = h->errCode;
    if (cell) *cell = h->errCell;
    if (particle) *particle = h->errParticle;
    if (msg && len) std::snprintf(msg, len, "%s", h->errMsg.c_str());
    return STORM_OK;
}

int storm_cuda_memory_bytes(StormHandle *h, uint64_t *bytes) {
    if (!h || !bytes) return STORM_ERR_INVALID_ARG;
    *bytes = h->memBytes;
    return STORM_OK;
}

int storm_cuda_launch_count(StormHandle *h, uint64_t *launches) {
    if (!h || !launches) return STORM_ERR_INVALID_ARG;
    *launches = h->launches;
    return STORM_OK;
}

int storm_cuda_set_profiling(StormHandle *h, int on) {
    if (!h) return STORM_ERR_INVALID_ARG;
    h->profiling = on != 0;
    return STORM_OK;
}

int storm_cuda_transport_timing(StormHandle *h, double *ms, uint64_t *launches, uint64_t *segments, int reset) {
    if (!h) return STORM_ERR_INVALID_ARG;
    if (ms) *ms = h->profMs;
    if (launches) *launches = h->profLaunches;
    if (segments) *segments = h->profSegments;
    if (reset) {
        h->profMs = 0.0;
        h->profLaunches = 0;
        h->profSegments = 0;
    }
    return STORM_OK;
}

int storm_cuda_autotune_transport(StormHandle *h, uint32_t steps_per_candidate) {
    if (!h || steps_per_candidate > 1000) return STORM_ERR_INVALID_ARG;
    h->tune = {};
    if (steps_per_candidate == 0) return STORM_OK;
    h->refill = true;
    h->tune.perCandidate = steps_per_candidate;
    h->burst = kTuneBursts[tune_candidate(0)];
    return STORM_OK;
}

int storm_cuda_transport_burst(StormHandle *h, uint32_t *burst, int *tuning) {
    if (!h || !burst || !tuning) return STORM_ERR_INVALID_ARG;
    *burst = h->burst;
    *tuning = h->tune.perCandidate ? 1 : 0;
    return STORM_OK;
}

int storm_cuda_set_transport_mode(StormHandle *h, int refill, uint32_t burst) {
    if (!h || burst == 0 || burst > 1024) return STORM_ERR_INVALID_ARG;
    h->refill = refill != 0;
    h->burst = burst;
    return STORM_OK;
}

int storm_cuda_set_transport_variant(StormHandle *h, int min_blocks_per_sm, int waves) {
    if (!h || min_blocks_per_sm < 1 || min_blocks_per_sm > 4 || waves < 1 || waves > 64) return STORM_ERR_INVALID_ARG;
    h->minBlocks = min_blocks_per_sm;
    int nb = transport_blocks_per_sm(h->minBlocks, h->fp32);
    h->transportGrid = static_cast<uint32_t>(h->smCount) * static_cast<uint32_t>(nb > 0 ? nb : 1) * waves;
    return STORM_OK;
}

int storm_cuda_set_segments_per_visit(StormHandle *h, uint32_t k) {
    if (!h || k == 0) return STORM_ERR_INVALID_ARG;
    h->K = k;
    return STORM_OK;
}

}  // extern "C"
