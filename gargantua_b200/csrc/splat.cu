// Splat pass (splat.metal:16-120): cloud-in-cell deposit of every particle
// into six 32-bit fixed-point sums per voxel, then a resolve of the sums into
// two rgba16f 3-D textures that also zeroes the sums for the next frame.
//
// Sums layout: one 24-byte record per voxel, interleaved (energy u32,
// energy*T u32, momentum x/y/z i32, mass u32), voxel index (z n + y) n + x.
// A corner's six atomics land in one or two 32-byte sectors, and the resolve
// reads and clears a warp's 32 records as 768 contiguous bytes.
//
// Integer sums are order-independent, so the grids are bit-exact whatever
// order the atomics arrive in, as long as each corner's fixed-point values
// are: this translation unit is built with --fmad=false and evaluates every
// float expression in the order the CPU replica (oracle/replica.c) does.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/gargantua_detmath.h"
#include "common.cuh"
#include "runtime.h"

namespace gg {

constexpr float ENERGY_FIXED = 16777216.0f;  // 2^24
constexpr float ENERGY_T_FIXED = 1048576.0f; // 2^20
constexpr float MOMENTUM_FIXED = 4096.0f;    // 2^12
constexpr float MASS_FIXED = 256.0f;         // 2^8

// Other ranks' copies of the sums (gg_volume_attach_peers), opened from
// their IPC handles: every word deposited here is added into each of them at
// the same offset, so the deposit is also the all-reduce.
struct PeerSums {
    uint32_t* sums[GG_MAX_PEERS];
    uint32_t count;
};

// One word into the sums and into every peer's copy.
__device__ __forceinline__ void add_word(uint32_t* sums, const PeerSums& peers, uint64_t offset, uint32_t v) {
    atomicAdd(sums + offset, v);
    if (peers.count != 0u) {
#pragma unroll
        for (uint32_t p = 0; p < GG_MAX_PEERS; ++p)
            if (p < peers.count) atomicAdd(peers.sums[p] + offset, v);
    }
}

struct SplatArgs {
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    uint32_t* __restrict__ sums;
    SplatUniforms u;
    uint32_t first_index;  // global index of slot 0, for the stochastic pick
    PeerSums peers;
};

// A particle's cloud-in-cell footprint (splat.metal:44-70): positions mapped
// to voxel-centre space of a cube of half extent u.halfExtent, the low and
// high corner of each axis, the fractional offsets, and the energy terms.
struct Footprint {
    int lx, ly, lz, hx, hy, hz;
    float fx, fy, fz, energy, relative;
};

__device__ __forceinline__ bool footprint(float4 p, const SplatUniforms& u, Footprint& f) {
    float ux = (p.x + u.halfExtent) / (2.0f * u.halfExtent);
    float uy = (p.y + u.halfExtent) / (2.0f * u.halfExtent);
    float uz = (p.z + u.halfExtent) / (2.0f * u.halfExtent);
    if (ux < 0.0f || uy < 0.0f || uz < 0.0f || ux >= 1.0f || uy >= 1.0f || uz >= 1.0f) return false;
    f.relative = p.w / u.peakTemperature;
    f.energy = f.relative * f.relative * f.relative * f.relative * u.emissionScale;
    const int n = (int)u.volumeSize;
    float gx = ux * (float)n - 0.5f, gy = uy * (float)n - 0.5f, gz = uz * (float)n - 0.5f;
    float bx = floorf(gx), by = floorf(gy), bz = floorf(gz);
    f.fx = gx - bx;
    f.fy = gy - by;
    f.fz = gz - bz;
    int lx = (int)bx, ly = (int)by, lz = (int)bz;
    f.hx = min(lx + 1, n - 1);
    f.hy = min(ly + 1, n - 1);
    f.hz = min(lz + 1, n - 1);
    f.lx = max(lx, 0);
    f.ly = max(ly, 0);
    f.lz = max(lz, 0);
    return true;
}

// One corner's six fixed-point values (splat.metal:25-37): energy, energy *
// T, momentum x/y/z, mass.
struct Deposit {
    uint32_t w[6];
};

__device__ __forceinline__ Deposit deposit_values(float weight, float energy, float relative, float vx, float vy,
                                                  float vz) {
    Deposit d;
    d.w[0] = (uint32_t)(energy * weight * ENERGY_FIXED + 0.5f);
    d.w[1] = (uint32_t)(energy * relative * weight * ENERGY_T_FIXED + 0.5f);
    float ms = weight * MOMENTUM_FIXED;
    d.w[2] = (uint32_t)(int32_t)rintf(vx * ms);
    d.w[3] = (uint32_t)(int32_t)rintf(vy * ms);
    d.w[4] = (uint32_t)(int32_t)rintf(vz * ms);
    d.w[5] = (uint32_t)(weight * MASS_FIXED + 0.5f);
    return d;
}

// The corners a particle deposits into: exact mode all eight with trilinear
// weights (w <= 0 skipped), stochastic mode one corner drawn with those
// weights as probabilities from pcg4d(global index, frame, seed), weight 1.
// Calls emit(x, y, z, weight) per corner.
template <typename Emit>
__device__ __forceinline__ void for_each_corner(const Footprint& f, const SplatUniforms& u, uint32_t global_index,
                                                Emit emit) {
    if (u.exactDeposit != 0u) {
#pragma unroll
        for (uint32_t c = 0; c < CIC_CORNERS; ++c) {
            bool bxs = (c & 1u) != 0u, bys = (c & 2u) != 0u, bzs = (c & 4u) != 0u;
            float wx = bxs ? f.fx : 1.0f - f.fx;
            float wy = bys ? f.fy : 1.0f - f.fy;
            float wz = bzs ? f.fz : 1.0f - f.fz;
            float w = wx * wy * wz;
            if (w <= 0.0f) continue;
            emit(bxs ? f.hx : f.lx, bys ? f.hy : f.ly, bzs ? f.hz : f.lz, w);
        }
    } else {
        uint4 h = pcg4d(make_uint4(global_index, u.frame, u.seed.x, u.seed.y));
        emit(unit_float(h.x) < f.fx ? f.hx : f.lx, unit_float(h.y) < f.fy ? f.hy : f.ly,
             unit_float(h.z) < f.fz ? f.hz : f.lz, 1.0f);
    }
}

// splatParticles (splat.metal:44-88), one thread per particle, six global
// atomics per corner straight into the sums (and into each peer's copy).
__global__ void __launch_bounds__(256) bin_kernel(SplatArgs a) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const SplatUniforms& u = a.u;
    if (i >= u.particleCount) return;
    Footprint f;
    if (!footprint(a.pos[i], u, f)) return;
    const float4 v = a.vel[i];
    const uint32_t n = u.volumeSize;
    for_each_corner(f, u, a.first_index + i, [&](int x, int y, int z, float w) {
        Deposit d = deposit_values(w, f.energy, f.relative, v.x, v.y, v.z);
        const uint64_t rec = 6ull * (((uint32_t)z * n + (uint32_t)y) * n + (uint32_t)x);
#pragma unroll
        for (int k = 0; k < 6; ++k) add_word(a.sums, a.peers, rec + k, d.w[k]);
    });
}

// ---------------------------------------------------------------------------
// Brick-privatised splat. The grid is cut into bricks of B^3 voxels; a
// particle belongs to the brick holding its low corner, so its eight corners
// fall in that brick's (B+1)^3 tile. Four launches:
//   count    each particle's brick (its key) and its place in a per-block
//            shared histogram of keys; each block adds its histogram to the
//            global counts with one atomic per brick, whose old value is the
//            block's first place in that brick, so every particle's place in
//            its brick (its rank) is stored with its key;
//   scan     one block: brick offsets and the work items, ceil(count /
//            chunk) chunks of each brick's sorted range, listed in a table;
//   scatter  each particle's index written at its brick's offset plus its
//            rank: brick order, with no atomics;
//   deposit  persistent blocks taking work items from a counter: the tile's
//            records (six words and a pad, see kTileStride) in shared
//            memory, the chunk's particles deposited there with shared
//            atomics, the non-zero words added to the sums (and to each
//            peer's copy) with one global atomic each and zeroed for the
//            next item.
// Integer sums do not depend on the order of the adds, so the grid equals
// the direct kernel's bit for bit.

constexpr uint32_t kBrickBlock = 256;
constexpr uint32_t kBrickParticlesPerBlock = 2048;  // count range of one block
constexpr uint32_t kOutside = 0xFFFFFFFFu;          // key of a particle outside the cube
constexpr uint32_t kMaxBricks = 32768;               // histogram of 128 KB shared memory

struct BrickArgs {
    const float4* __restrict__ pos;
    const float4* __restrict__ vel;
    uint32_t* __restrict__ sums;
    SplatUniforms u;
    uint32_t first_index;
    uint32_t edge;       // B
    uint32_t edge_shift; // log2(B)
    uint32_t per_axis;   // ceil(n / B)
    uint32_t bricks;     // per_axis^3
    uint32_t chunk;      // particles per deposit work item
    uint32_t chunk_shift;  // log2(chunk) when chunk is a power of two, else 32
    uint32_t* counts;    // [kMaxBricks], zero between calls (the scan re-zeroes what it read)
    uint32_t* offsets;   // [bricks + 1], exclusive scan of counts
    uint32_t* items;     // [bricks + 1], exclusive scan of ceil(count / chunk)
    uint32_t* sorted;    // [particleCount], particle slots in brick order
    uint32_t* keys;      // [particleCount], each particle's brick (kOutside: none), from the count pass
    uint32_t* ranks;     // [particleCount], each particle's place in its brick, from the count pass
    uint4* work;         // [max_items], per work item: brick, first and end sorted slot (from the scan)
    uint32_t max_items;  // ceil(particleCount / chunk) + bricks, a bound on the work items
    uint32_t* next;      // the deposit blocks' work counter (zeroed by the scan)
    PeerSums peers;
};

__device__ __forceinline__ uint32_t brick_of(const Footprint& f, const BrickArgs& a) {
    return (((uint32_t)f.lz >> a.edge_shift) * a.per_axis + ((uint32_t)f.ly >> a.edge_shift)) * a.per_axis +
           ((uint32_t)f.lx >> a.edge_shift);
}

// Inclusive sum over the warp of a value per lane (shuffle scan).
__device__ __forceinline__ uint32_t warp_inclusive(uint32_t v, uint32_t lane) {
#pragma unroll
    for (uint32_t off = 1; off < 32u; off <<= 1) {
        uint32_t u = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += u;
    }
    return v;
}

// Work items of a brick of c particles: ceil(c / chunk), a shift when the
// chunk is a power of two.
__device__ __forceinline__ uint32_t brick_items(uint32_t c, const BrickArgs& a) {
    return a.chunk_shift < 32u ? (c + a.chunk - 1u) >> a.chunk_shift : (c + a.chunk - 1u) / a.chunk;
}

// Exclusive scans of the brick counts (offsets) and of their work
// items (items), by one block of kScanThreads threads: each thread scans a
// contiguous run of bricks, loading its counts kScanBatch at a time so the
// loads are in flight together; the per-thread totals are scanned with warp
// shuffles and one pass over the warp totals. The counts are zeroed behind
// the read, so they start at zero at the next call. (Run by the count
// kernel's last block instead, the scan's registers cost the count pass its
// occupancy: 31 -> 56 us at 256^3.)
constexpr uint32_t kScanBatch = 8;
constexpr uint32_t kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) brick_scan_kernel(BrickArgs a) {
    constexpr uint32_t kWarps = kScanThreads / 32u;
    __shared__ uint32_t warp_p[kWarps], warp_i[kWarps];
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t per = (a.bricks + kScanThreads - 1u) / kScanThreads;
    const uint32_t b0 = min(threadIdx.x * per, a.bricks), b1 = min(b0 + per, a.bricks);
    uint32_t sp = 0, si = 0;
    for (uint32_t b = b0; b < b1; b += kScanBatch) {
        uint32_t c[kScanBatch];
#pragma unroll
        for (uint32_t j = 0; j < kScanBatch; ++j) c[j] = b + j < b1 ? a.counts[b + j] : 0u;
#pragma unroll
        for (uint32_t j = 0; j < kScanBatch; ++j) {
            sp += c[j];
            si += brick_items(c[j], a);
        }
    }
    const uint32_t ip = warp_inclusive(sp, lane), ii = warp_inclusive(si, lane);
    if (lane == 31u) {
        warp_p[warp] = ip;
        warp_i[warp] = ii;
    }
    __syncthreads();
    if (warp == 0) {
        const uint32_t wp = warp_inclusive(lane < kWarps ? warp_p[lane] : 0u, lane);
        const uint32_t wi = warp_inclusive(lane < kWarps ? warp_i[lane] : 0u, lane);
        if (lane < kWarps) {
            warp_p[lane] = wp;  // inclusive totals through warp `lane`
            warp_i[lane] = wi;
        }
    }
    __syncthreads();
    uint32_t op = (warp ? warp_p[warp - 1] : 0u) + ip - sp;  // exclusive prefix of this thread's run
    uint32_t oi = (warp ? warp_i[warp - 1] : 0u) + ii - si;
    for (uint32_t b = b0; b < b1; b += kScanBatch) {
        uint32_t c[kScanBatch];
#pragma unroll
        for (uint32_t j = 0; j < kScanBatch; ++j) c[j] = b + j < b1 ? a.counts[b + j] : 0u;
#pragma unroll
        for (uint32_t j = 0; j < kScanBatch; ++j) {
            if (b + j >= b1) break;
            a.counts[b + j] = 0u;
            a.offsets[b + j] = op;
            a.items[b + j] = oi;
            // The brick's work items: consecutive chunks of its sorted range.
            for (uint32_t s = 0; s < c[j];) {
                const uint32_t len = min(c[j] - s, a.chunk);
                if (oi < a.max_items) a.work[oi] = make_uint4(b + j, op + s, op + s + len, 0u);
                ++oi;
                s += len;
            }
            op += c[j];
        }
    }
    if (threadIdx.x == kScanThreads - 1u) {
        a.offsets[a.bricks] = warp_p[kWarps - 1];
        a.items[a.bricks] = warp_i[kWarps - 1];
        *a.next = 0u;
    }
}

// Each block histograms its particles' bricks in shared memory and adds the
// histogram to the counts.
// Each thread's particles in the count pass: their loads are issued
// together before any is used, so a thread waits for memory once, not once
// per particle.
constexpr uint32_t kPerThread = kBrickParticlesPerBlock / kBrickBlock;
static_assert(kBrickParticlesPerBlock % kBrickBlock == 0, "count ranges split evenly over a block");

__global__ void __launch_bounds__(kBrickBlock) brick_count_kernel(BrickArgs a) {
    extern __shared__ uint32_t hist[];
    const uint32_t first = blockIdx.x * kBrickParticlesPerBlock + threadIdx.x;
    float4 p[kPerThread];
#pragma unroll
    for (uint32_t j = 0; j < kPerThread; ++j) {
        const uint32_t i = first + j * kBrickBlock;
        if (i < a.u.particleCount) p[j] = a.pos[i];
    }
    for (uint32_t b = threadIdx.x; b < a.bricks; b += blockDim.x) hist[b] = 0u;
    __syncthreads();
    uint32_t key[kPerThread], rank[kPerThread];
#pragma unroll
    for (uint32_t j = 0; j < kPerThread; ++j) {
        key[j] = kOutside;
        rank[j] = 0u;
        Footprint f;
        if (first + j * kBrickBlock < a.u.particleCount && footprint(p[j], a.u, f)) {
            key[j] = brick_of(f, a);
            rank[j] = atomicAdd(&hist[key[j]], 1u);  // place among this block's particles of the brick
        }
    }
    __syncthreads();
    // The block's histogram into the counts; each old count is where the
    // block's particles of that brick start.
    for (uint32_t b = threadIdx.x; b < a.bricks; b += blockDim.x)
        if (hist[b]) hist[b] = atomicAdd(&a.counts[b], hist[b]);
    __syncthreads();
#pragma unroll
    for (uint32_t j = 0; j < kPerThread; ++j) {
        const uint32_t i = first + j * kBrickBlock;
        if (i >= a.u.particleCount) break;
        a.keys[i] = key[j];
        if (key[j] != kOutside) a.ranks[i] = hist[key[j]] + rank[j];
    }
}

// One particle per thread: its index at its brick's offset plus its rank.
__global__ void __launch_bounds__(kBrickBlock) brick_scatter_kernel(BrickArgs a) {
    const uint32_t i = blockIdx.x * kBrickBlock + threadIdx.x;
    if (i >= a.u.particleCount) return;
    const uint32_t key = a.keys[i];
    if (key >= a.bricks) return;
    const uint32_t slot = a.offsets[key] + a.ranks[i];
    if (slot < a.u.particleCount) a.sorted[slot] = i;  // always: ranks and offsets came from the same counts
}

// Words per record in the deposit's shared tile: the six sums and one pad
// word. With an odd stride the same word of records at random cells falls
// on all 32 banks; with stride 6, 6 cell + c is even-offset and a warp's
// atomics to one word reach only 16 banks, twice the conflicts.
constexpr uint32_t kTileStride = 7;

// Threads of a deposit block. A 16^3 brick's 17^3 tile of seven-word records
// takes 138 KB of shared memory, so one block fills an SM: it gets 1024 threads to keep enough
// shared atomics in flight; the smaller tiles fit several 256-thread blocks.
template <uint32_t B> constexpr uint32_t deposit_threads() { return B == 16u ? 1024u : kBrickBlock; }
// Resident blocks asked of the compiler: 64 registers a thread at most.
template <uint32_t B> constexpr uint32_t deposit_min_blocks() { return B == 16u ? 1u : 4u; }

// Persistent deposit: as many blocks as fit on the device at once, each
// zeroing its tile once and then taking work items from a counter until none
// is left. Per item:
//   deposit  the chunk's particles added into the tile with shared atomics,
//            and the y and z range of their low corners kept (warp minimum
//            and maximum, one shared atomic per warp);
//   flush    the tile rows inside that range (a row is T cells along x, 6 T
//            words, contiguous in the sums as well), one warp per row: each
//            non-zero word is added to the sums (and to each attached
//            peer's copy) with one global atomic and zeroed again in the
//            tile, so the next item finds a zero tile.
// Cells outside the range hold no deposit: a particle's corners lie at its
// low corner or one voxel above it on each axis.
template <uint32_t B>
__global__ void __launch_bounds__(deposit_threads<B>(), deposit_min_blocks<B>()) brick_deposit_kernel(BrickArgs a) {
    constexpr uint32_t T = B + 1;
    constexpr uint32_t kCells = T * T * T;
    constexpr uint32_t kRowWords = 6u * T;
    constexpr uint32_t kRowSteps = (kRowWords + 31u) / 32u;
    extern __shared__ uint32_t tile[];
    __shared__ uint4 job;
    __shared__ uint32_t range[4];  // low corners' y min, y max, z min, z max in the tile
    for (uint32_t w = threadIdx.x; w < kCells * kTileStride; w += blockDim.x) tile[w] = 0u;
    const uint32_t total = min(a.items[a.bricks], a.max_items);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, warps = blockDim.x >> 5;
    const uint32_t n = a.u.volumeSize;
    // Every pass takes one counter value, so a block makes at most total + 1.
    for (uint32_t pass = 0; pass <= total; ++pass) {
        if (threadIdx.x == 0) {
            const uint32_t k = atomicAdd(a.next, 1u);
            job = k < total ? a.work[k] : make_uint4(kOutside, 0u, 0u, 0u);
            range[0] = range[2] = B;
            range[1] = range[3] = 0u;
        }
        __syncthreads();  // also puts the previous item's flush before this item's adds
        const uint4 item = job;
        if (item.x >= a.bricks) break;  // no work left: the same for every thread
        const uint32_t b = item.x, begin = item.y, end = item.z;
        const uint32_t bx = b % a.per_axis, by = (b / a.per_axis) % a.per_axis, bz = b / (a.per_axis * a.per_axis);
        const int ox = (int)(bx * B), oy = (int)(by * B), oz = (int)(bz * B);
        uint32_t ylo = B, yhi = 0u, zlo = B, zhi = 0u;
        // One particle per thread per pass. Loading four before depositing
        // any (to overlap their gathers) ran slower: 257 against 232 us for
        // 4M particles into 16^3 bricks of a 256^3 grid, 86 against 82 us
        // for 1M into 8^3 bricks of 128^3.
        for (uint32_t k = begin + threadIdx.x; k < end; k += blockDim.x) {
            const uint32_t slot = a.sorted[k];
            const float4 p = a.pos[slot];
            Footprint f;
            // Always inside and in this brick (the count pass put it
            // here); the test keeps every tile index in bounds regardless.
            if (!footprint(p, a.u, f)) continue;
            const uint32_t ty = (uint32_t)(f.ly - oy), tz = (uint32_t)(f.lz - oz);
            if ((uint32_t)(f.lx - ox) >= B || ty >= B || tz >= B) continue;
            ylo = min(ylo, ty);
            yhi = max(yhi, ty);
            zlo = min(zlo, tz);
            zhi = max(zhi, tz);
            const float4 v = a.vel[slot];
            if (a.u.exactDeposit != 0u) {
                // All eight corners, their values first and then their 48
                // adds back to back. A corner of weight 0 adds zeros, the
                // same sums as skipping it.
                uint32_t* low = tile + kTileStride * ((tz * T + ty) * T + (uint32_t)(f.lx - ox));
                const uint32_t sx = kTileStride * (uint32_t)(f.hx - f.lx);
                const uint32_t sy = kTileStride * T * (uint32_t)(f.hy - f.ly);
                const uint32_t sz = kTileStride * T * T * (uint32_t)(f.hz - f.lz);
                Deposit d[CIC_CORNERS];
#pragma unroll
                for (uint32_t c = 0; c < CIC_CORNERS; ++c) {
                    const float wx = (c & 1u) ? f.fx : 1.0f - f.fx;
                    const float wy = (c & 2u) ? f.fy : 1.0f - f.fy;
                    const float wz = (c & 4u) ? f.fz : 1.0f - f.fz;
                    d[c] = deposit_values(wx * wy * wz, f.energy, f.relative, v.x, v.y, v.z);
                }
#pragma unroll
                for (uint32_t c = 0; c < CIC_CORNERS; ++c) {
                    uint32_t* rec = low + ((c & 1u) ? sx : 0u) + ((c & 2u) ? sy : 0u) + ((c & 4u) ? sz : 0u);
#pragma unroll
                    for (int q = 0; q < 6; ++q) atomicAdd(rec + q, d[c].w[q]);
                }
            } else {
                for_each_corner(f, a.u, a.first_index + slot, [&](int x, int y, int z, float w) {
                    Deposit d = deposit_values(w, f.energy, f.relative, v.x, v.y, v.z);
                    uint32_t* rec = tile + kTileStride * (((uint32_t)(z - oz) * T + (uint32_t)(y - oy)) * T +
                                                          (uint32_t)(x - ox));
#pragma unroll
                    for (int q = 0; q < 6; ++q) atomicAdd(rec + q, d.w[q]);
                });
            }
        }
        ylo = __reduce_min_sync(0xffffffffu, ylo);
        yhi = __reduce_max_sync(0xffffffffu, yhi);
        zlo = __reduce_min_sync(0xffffffffu, zlo);
        zhi = __reduce_max_sync(0xffffffffu, zhi);
        if (lane == 0u) {
            atomicMin(&range[0], ylo);
            atomicMax(&range[1], yhi);
            atomicMin(&range[2], zlo);
            atomicMax(&range[3], zhi);
        }
        __syncthreads();
        const uint32_t y0 = range[0], z0 = range[2];
        const uint32_t rows_y = range[1] >= y0 ? range[1] + 2u - y0 : 0u;  // low rows and the row above the last
        const uint32_t rows_z = range[3] >= z0 ? range[3] + 2u - z0 : 0u;
        for (uint32_t r = warp; r < rows_y * rows_z; r += warps) {
            const uint32_t ry = y0 + r % rows_y, rz = z0 + r / rows_y;
            const uint32_t y = (uint32_t)oy + ry, z = (uint32_t)oz + rz;
            uint32_t* row = tile + kTileStride * ((rz * T + ry) * T);
            const uint64_t dst = 6ull * (((uint64_t)z * n + y) * n + (uint32_t)ox);
#pragma unroll
            for (uint32_t s = 0; s < kRowSteps; ++s) {
                const uint32_t w = lane + 32u * s;
                if (w >= kRowWords) break;
                const uint32_t cx = w / 6u, c = w - cx * 6u;
                uint32_t* word = row + kTileStride * cx + c;
                const uint32_t val = *word;
                if (val == 0u) continue;
                *word = 0u;
                if ((uint32_t)ox + cx < n && y < n && z < n) add_word(a.sums, a.peers, dst + w, val);
            }
        }
        __syncthreads();
    }
}

template <uint32_t B> constexpr uint32_t tile_bytes() { return (B + 1) * (B + 1) * (B + 1) * kTileStride * 4u; }

struct ResolveArgs {
    uint32_t* __restrict__ sums;
    cudaSurfaceObject_t emission;
    cudaSurfaceObject_t velocity;
    const float4* __restrict__ blackbody;
    SplatUniforms u;
    double log_t_min, log_t_max;  // gg_log_d of the blackbody range, the same values on every device and host
    uint32_t clear_mask;          // 0: the clear stores loaded & 0 (see resolve_kernel)
};

// Blackbody coordinate (Common.h:56-59) in double with the shared series
// log, rounded once, so the resolve's bits match the CPU replica's.
__device__ __forceinline__ float bb_coordinate_det(float temperature, double lo, double hi) {
    float t = fminf(fmaxf(temperature, BLACKBODY_T_MIN), BLACKBODY_T_MAX);
    return (float)((gg_log_d((double)t) - lo) / (hi - lo));
}

// resolveVolume (splat.metal:93-120) fused with the clear of the sums
// (Volume.swift:34-43): each voxel's record is read once and written back
// as zeros. The zeros are the loaded words ANDed with a mask of 0 passed at
// launch, so each store waits for its own load: a store issued while the
// read of its line is still in flight runs about 9x slower on B200 (a
// 403 MB read-and-zero pass measured 0.73 TB/s that way, 6.3 TB/s with the
// stores after the data). Rows come from the grid's y and z (no index
// divisions).

// One voxel's record (E, E T, px, py, pz, mass) to its two texels.
__device__ __forceinline__ void resolve_voxel(const ResolveArgs& a, uint32_t e, uint32_t et, uint32_t px, uint32_t py,
                                              uint32_t pz, uint32_t mass, float inverse_volume, uint32_t x, uint32_t y,
                                              uint32_t z) {
    float count = (float)mass / MASS_FIXED;
    float energy = (float)e / ENERGY_FIXED;
    float energy_t = (float)et / ENERGY_T_FIXED;
    float tr = 0.0f, tg = 0.0f, tb = 0.0f;
    if (energy > 0.0f) {
        float mean_t = energy_t / energy * a.u.peakTemperature;
        float c = bb_coordinate_det(mean_t, a.log_t_min, a.log_t_max) * (float)BLACKBODY_TABLE_SIZE - 0.5f;
        float fl = floorf(c);
        float f = c - fl;
        int i0 = (int)fl, i1 = i0 + 1;
        i0 = min(max(i0, 0), (int)BLACKBODY_TABLE_SIZE - 1);
        i1 = min(max(i1, 0), (int)BLACKBODY_TABLE_SIZE - 1);
        float4 ta = __ldg(a.blackbody + i0), tb4 = __ldg(a.blackbody + i1);
        tr = ta.x + (tb4.x - ta.x) * f;
        tg = ta.y + (tb4.y - ta.y) * f;
        tb = ta.z + (tb4.z - ta.z) * f;
    }
    float mx = (float)(int32_t)px / MOMENTUM_FIXED;
    float my = (float)(int32_t)py / MOMENTUM_FIXED;
    float mz = (float)(int32_t)pz / MOMENTUM_FIXED;
    float density = count * inverse_volume;
    float vx = count > 0.0f ? mx / count : 0.0f;
    float vy = count > 0.0f ? my / count : 0.0f;
    float vz = count > 0.0f ? mz / count : 0.0f;
    surf3Dwrite(pack_half4(tr * energy * inverse_volume, tg * energy * inverse_volume, tb * energy * inverse_volume,
                           density),
                a.emission, x * 8, y, z);
    surf3Dwrite(pack_half4(vx, vy, vz, 1.0f), a.velocity, x * 8, y, z);
}

__device__ __forceinline__ float resolve_inverse_volume(const ResolveArgs& a) {
    float voxel = 2.0f * a.u.halfExtent / (float)a.u.volumeSize;
    return 1.0f / (voxel * voxel * voxel);
}

// One voxel per thread; a block is 32 consecutive voxels of each of 8
// neighbouring rows. Against 128 voxels of one row per block this ran the
// 256^3 resolve in 203 us instead of 252 (the surface stores of a block land
// in fewer tiles of the block-linear texture layout); four voxels per thread
// were slower at 128^3 (fewer waves of blocks) and no faster at 256^3, and
// two neighbouring voxels per thread with 16-byte record loads and clearing
// stores slower at both (38.6 against 30.9 us at 128^3, 255 against 210 at
// 256^3).
constexpr uint32_t kResolveRows = 8;

__global__ void __launch_bounds__(32 * kResolveRows) resolve_kernel(ResolveArgs a) {
    const uint32_t n = a.u.volumeSize;
    const uint32_t x = blockIdx.x * 32u + threadIdx.x, y = blockIdx.y * kResolveRows + threadIdx.y, z = blockIdx.z;
    if (x >= n || y >= n) return;
    const uint64_t index = ((uint64_t)z * n + y) * n + x;
    uint2* rec = reinterpret_cast<uint2*>(a.sums + 6ull * index);
    uint2 r0 = rec[0], r1 = rec[1], r2 = rec[2];
    const uint32_t m = a.clear_mask;
    rec[0] = make_uint2(r0.x & m, r0.y & m);
    rec[1] = make_uint2(r1.x & m, r1.y & m);
    rec[2] = make_uint2(r2.x & m, r2.y & m);
    resolve_voxel(a, r0.x, r0.y, r1.x, r1.y, r2.x, r2.y, resolve_inverse_volume(a), x, y, z);
}

__global__ void clear_kernel(uint4* sums, uint64_t count16) {
    uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count16) sums[i] = make_uint4(0u, 0u, 0u, 0u);
}

}  // namespace gg

using namespace gg;

static uint32_t bricks_per_axis(uint32_t size, uint32_t edge) { return (size + edge - 1u) / edge; }

// Shapes gg_splat_bin runs: edge 0 (direct), or 4, 8, 16 with a positive
// chunk and at most kMaxBricks bricks.
static int check_shape(const gg_volume* vol, uint32_t edge, uint32_t chunk) {
    if (edge == 0u) return GG_OK;
    if (edge != 4u && edge != 8u && edge != 16u)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Brick edge %u is not 0, 4, 8 or 16.", edge);
    if (chunk == 0u || chunk > (1u << 24))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "Chunk %u is outside 1..16777216 particles.", chunk);
    const uint64_t per = bricks_per_axis(vol->size, edge);
    if (per * per * per > kMaxBricks)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "A %u^3 volume in %u^3 bricks makes %llu bricks, over %u.", vol->size,
                        edge, (unsigned long long)(per * per * per), kMaxBricks);
    return GG_OK;
}

// Opt the kernels that need more than 48 KB of dynamic shared memory in,
// once per device.
static int allow_shared(const void* kernel, int bytes, int device, int slot) {
    static std::mutex mu;
    static int done[64][5] = {};
    if (bytes <= 48 * 1024 || device >= 64) return GG_OK;
    std::lock_guard<std::mutex> lock(mu);
    if (done[device][slot] >= bytes) return GG_OK;
    GG_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes), "shared memory opt-in");
    done[device][slot] = bytes;
    return GG_OK;
}

static uint64_t align256(uint64_t x) { return (x + 255u) & ~255ull; }

static PeerSums peer_sums(const gg_volume* vol) {
    PeerSums p{};
    p.count = vol->peers;
    for (uint32_t k = 0; k < vol->peers && k < GG_MAX_PEERS; ++k) p.sums[k] = vol->peer_sums[k];
    return p;
}

static void close_peers(gg_volume* vol) {
    for (uint32_t k = 0; k < vol->peers && k < GG_MAX_PEERS; ++k)
        if (vol->peer_sums[k]) cudaIpcCloseMemHandle(vol->peer_sums[k]);
    for (uint32_t k = 0; k < GG_MAX_PEERS; ++k) vol->peer_sums[k] = nullptr;
    vol->peers = 0;
}

// The persistent deposit's grid: the blocks of brick_deposit_kernel<B> that
// are resident at once on the device (its occupancy with its tile, found
// once per device), at most one per work item.
template <uint32_t B> static int launch_deposit(gg_context* ctx, const BrickArgs& a) {
    constexpr int kSlot = B == 4u ? 0 : B == 8u ? 1 : 2;
    static std::mutex mu;
    static int resident[64][3] = {};
    const int smem = (int)tile_bytes<B>();
    const void* kernel = (const void*)brick_deposit_kernel<B>;
    GG_CHECK(allow_shared(kernel, smem, ctx->device, 2 + kSlot));
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(mu);
        if (ctx->device < 64) per_sm = resident[ctx->device][kSlot];
        if (per_sm == 0) {
            GG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, (int)deposit_threads<B>(), smem),
                    "deposit occupancy");
            if (per_sm < 1) per_sm = 1;
            if (ctx->device < 64) resident[ctx->device][kSlot] = per_sm;
        }
    }
    const uint64_t grid = std::min<uint64_t>(a.max_items, (uint64_t)per_sm * (uint64_t)ctx->sm_count);
    brick_deposit_kernel<B><<<(uint32_t)std::max<uint64_t>(grid, 1u), deposit_threads<B>(), smem, ctx->stream>>>(a);
    return GG_OK;
}

// gg_splat_bin with an explicit shape (caller holds the context lock and has
// checked the arguments).
static int splat_bin_shaped(gg_particles* ps, gg_volume* vol, const SplatUniforms* u, uint32_t edge, uint32_t chunk) {
    gg_context* ctx = vol->ctx;
    if (edge == 0u) {
        SplatArgs a{ps->pos, ps->vel, vol->sums, *u, ps->first_index, peer_sums(vol)};
        bin_kernel<<<(ps->count + 255u) / 256u, 256, 0, ctx->stream>>>(a);
        return gg::launch_status("splat bin");
    }
    GG_CHECK(check_shape(vol, edge, chunk));
    const uint32_t per = bricks_per_axis(vol->size, edge);
    const uint32_t bricks = per * per * per;
    // counts (a fixed kMaxBricks words, whatever the shape, so that the
    // zeros the scan leaves behind stay counts), offsets, items, sorted
    // slots, keys, ranks.
    const uint64_t counts_bytes = align256(4ull * kMaxBricks);
    const uint64_t words = counts_bytes + align256(4ull * (bricks + 1u)) * 2u;
    // Work items number at most ceil(count / chunk) + one per non-empty brick.
    const uint64_t max_items = ((uint64_t)ps->count + chunk - 1u) / chunk + bricks;
    if (max_items >= 0xFFFFFFFFull) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Too many splat work items.");
    const uint64_t tail = words + 3u * align256(4ull * ps->count);  // work table, then the work counter
    const uint64_t bytes = tail + align256(16ull * max_items) + 256u;
    const uint64_t capacity_before = vol->brick_scratch_capacity;  // changes when the scratch is reallocated
    GG_CHECK(gg::ensure_capacity(ctx, &vol->brick_scratch, &vol->brick_scratch_capacity, bytes, "splat bricks"));
    char* base = static_cast<char*>(vol->brick_scratch);
    if (vol->brick_scratch_capacity != capacity_before || !vol->brick_counts_zero) {
        GG_CUDA(cudaMemsetAsync(base, 0, counts_bytes, ctx->stream), "brick counts");
        vol->brick_counts_zero = true;
    }
    BrickArgs a;
    a.peers = peer_sums(vol);
    a.pos = ps->pos;
    a.vel = ps->vel;
    a.sums = vol->sums;
    a.u = *u;
    a.first_index = ps->first_index;
    a.edge = edge;
    a.edge_shift = edge == 4u ? 2u : edge == 8u ? 3u : 4u;  // check_shape admits 4, 8 and 16
    a.per_axis = per;
    a.bricks = bricks;
    a.chunk = chunk;
    a.chunk_shift = 32u;
    if ((chunk & (chunk - 1u)) == 0u)
        for (uint32_t k = 0; k < 32u; ++k)
            if ((1u << k) == chunk) a.chunk_shift = k;
    a.counts = reinterpret_cast<uint32_t*>(base);
    a.offsets = reinterpret_cast<uint32_t*>(base + counts_bytes);
    a.items = reinterpret_cast<uint32_t*>(base + counts_bytes + align256(4ull * (bricks + 1u)));
    a.sorted = reinterpret_cast<uint32_t*>(base + words);
    a.keys = reinterpret_cast<uint32_t*>(base + words + align256(4ull * ps->count));
    a.ranks = reinterpret_cast<uint32_t*>(base + words + 2u * align256(4ull * ps->count));
    a.work = reinterpret_cast<uint4*>(base + tail);
    a.max_items = (uint32_t)max_items;
    a.next = reinterpret_cast<uint32_t*>(base + tail + align256(16ull * max_items));
    const int hist = (int)(4u * bricks);
    GG_CHECK(allow_shared((const void*)brick_count_kernel, hist, ctx->device, 0));
    const uint32_t blocks = (ps->count + kBrickParticlesPerBlock - 1u) / kBrickParticlesPerBlock;
    // A failed launch leaves the counts in an unknown state: clear them next time.
    vol->brick_counts_zero = false;
    brick_count_kernel<<<blocks, kBrickBlock, hist, ctx->stream>>>(a);
    GG_CHECK(gg::launch_status("brick count"));
    brick_scan_kernel<<<1, kScanThreads, 0, ctx->stream>>>(a);
    GG_CHECK(gg::launch_status("brick scan"));
    vol->brick_counts_zero = true;
    brick_scatter_kernel<<<(ps->count + kBrickBlock - 1u) / kBrickBlock, kBrickBlock, 0, ctx->stream>>>(a);
    GG_CHECK(gg::launch_status("brick scatter"));
    if (edge == 4u) GG_CHECK(launch_deposit<4>(ctx, a));
    else if (edge == 8u) GG_CHECK(launch_deposit<8>(ctx, a));
    else GG_CHECK(launch_deposit<16>(ctx, a));
    return gg::launch_status("brick deposit");
}

static int check_splat(const gg_particles* ps, const gg_volume* vol, const SplatUniforms* u, const char* what) {
    if (!vol || !u) return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s needs a volume and uniforms.", what);
    if (u->volumeSize != vol->size)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: uniforms give a %u^3 volume but the volume is %u^3.", what,
                        u->volumeSize, vol->size);
    if (ps && u->particleCount != ps->count)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: uniforms give %u particles but the system has %u.", what,
                        u->particleCount, ps->count);
    if (ps && ps->ctx != vol->ctx) return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: handles from different contexts.", what);
    if (!(u->halfExtent > 0.0f) || !(u->peakTemperature > 0.0f))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "%s: halfExtent and peakTemperature must be positive.", what);
    return GG_OK;
}

extern "C" {

GG_API int gg_volume_create(gg_context* ctx, uint32_t size, gg_volume** out) {
    if (!ctx || !out) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_create needs a context and an output.");
    *out = nullptr;
    if (size < 2 || size > 1024) return gg::fail(GG_ERR_INVALID_ARGUMENT, "Volume size %u is outside 2..1024.", size);
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t voxels = (uint64_t)size * size * size;
    const uint64_t sums_bytes = voxels * 24u;
    const uint64_t tex_bytes = voxels * 8u * 2u;
    if (ctx->used + sums_bytes + tex_bytes > ctx->budget)
        return gg::fail(GG_ERR_OVER_BUDGET, "A %u^3 volume needs %llu bytes but the budget has %llu bytes left.", size,
                        (unsigned long long)(sums_bytes + tex_bytes), (unsigned long long)(ctx->budget - ctx->used));
    gg_volume* vol = new gg_volume();
    vol->ctx = ctx;
    vol->size = size;
    // Default shapes, from timing the shapes on the presets' settled disks
    // (250k/96^3, 1M/128^3, 4M/256^3, uniform and concentrated): the
    // stochastic deposit (one corner per particle) is fastest with direct
    // global atomics at every size; the exact one with 16^3 bricks from 96^3
    // up (41, 73 and 230 us against 45, 83 and 620 us with 8^3 bricks), in
    // chunks of 4096, 8192 and 16384 particles, and with 8^3 bricks below.
    vol->brick_edge[0] = 0u;
    vol->brick_chunk[0] = 0u;
    vol->brick_edge[1] = size >= 96u ? 16u : 8u;
    vol->brick_chunk[1] = size > 128u ? 16384u : size > 96u ? 8192u : size >= 96u ? 4096u : 1024u;
    int s = gg::device_alloc(ctx, sums_bytes, (void**)&vol->sums, "volume sums");
    if (s == GG_OK) s = gg::cuda_status(cudaMemsetAsync(vol->sums, 0, sums_bytes, ctx->stream), "volume clear");
    cudaChannelFormatDesc desc = cudaCreateChannelDescHalf4();
    cudaExtent extent = make_cudaExtent(size, size, size);
    if (s == GG_OK) s = gg::cuda_status(cudaMalloc3DArray(&vol->emission, &desc, extent, cudaArraySurfaceLoadStore), "emission volume");
    if (s == GG_OK) s = gg::cuda_status(cudaMalloc3DArray(&vol->velocity, &desc, extent, cudaArraySurfaceLoadStore), "velocity volume");
    if (s == GG_OK) ctx->used += tex_bytes;
    vol->bytes = sums_bytes + tex_bytes;
    for (int k = 0; k < 2 && s == GG_OK; ++k) {
        cudaArray_t arr = k == 0 ? vol->emission : vol->velocity;
        cudaResourceDesc res{};
        res.resType = cudaResourceTypeArray;
        res.res.array.array = arr;
        // Trilinear, normalized coordinates, zero outside (march.metal:18).
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
        td.filterMode = cudaFilterModeLinear;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 1;
        cudaTextureObject_t tex = 0;
        cudaSurfaceObject_t surf = 0;
        s = gg::cuda_status(cudaCreateTextureObject(&tex, &res, &td, nullptr), "volume texture");
        if (s == GG_OK) s = gg::cuda_status(cudaCreateSurfaceObject(&surf, &res), "volume surface");
        if (k == 0) { vol->emission_tex = tex; vol->emission_surf = surf; }
        else { vol->velocity_tex = tex; vol->velocity_surf = surf; }
    }
    if (s == GG_OK) {
        // Start with empty textures: a resolve of the zeroed sums.
        SplatUniforms u{};
        u.volumeSize = size;
        u.halfExtent = VOLUME_HALF_EXTENT;
        u.peakTemperature = T_PEAK_DEFAULT;
        s = gg_splat_resolve(vol, &u, nullptr);
    }
    if (s == GG_OK) s = gg::cuda_status(cudaStreamSynchronize(ctx->stream), "volume set-up");
    if (s != GG_OK) {
        gg_volume_destroy(vol);
        return s;
    }
    *out = vol;
    return GG_OK;
}

GG_API void gg_volume_destroy(gg_volume* vol) {
    if (!vol) return;
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    close_peers(vol);
    if (vol->emission_tex) cudaDestroyTextureObject(vol->emission_tex);
    if (vol->velocity_tex) cudaDestroyTextureObject(vol->velocity_tex);
    if (vol->emission_surf) cudaDestroySurfaceObject(vol->emission_surf);
    if (vol->velocity_surf) cudaDestroySurfaceObject(vol->velocity_surf);
    if (vol->emission) cudaFreeArray(vol->emission);
    if (vol->velocity) cudaFreeArray(vol->velocity);
    const uint64_t voxels = (uint64_t)vol->size * vol->size * vol->size;
    gg::device_free(ctx, vol->sums, voxels * 24u);
    gg::device_free(ctx, vol->brick_scratch, vol->brick_scratch_capacity);
    uint64_t tex = voxels * 16u;
    ctx->used -= tex < ctx->used ? tex : ctx->used;
    delete vol;
}

GG_API int gg_splat_bin(gg_particles* ps, gg_volume* vol, const SplatUniforms* u) {
    if (!ps) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_splat_bin needs a particle system.");
    GG_CHECK(check_splat(ps, vol, u, "gg_splat_bin"));
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const int mode = u->exactDeposit ? 1 : 0;
    return splat_bin_shaped(ps, vol, u, vol->brick_edge[mode], vol->brick_chunk[mode]);
}

GG_API int gg_volume_splat_shape(gg_volume* vol, int exact, uint32_t brick_edge, uint32_t chunk) {
    if (!vol) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_splat_shape needs a volume.");
    GG_CHECK(check_shape(vol, brick_edge, chunk));
    std::lock_guard<std::recursive_mutex> lock(vol->ctx->mu);
    vol->brick_edge[exact ? 1 : 0] = brick_edge;
    vol->brick_chunk[exact ? 1 : 0] = brick_edge ? chunk : 0u;
    return GG_OK;
}

GG_API int gg_splat_autotune(gg_particles* ps, gg_volume* vol, const SplatUniforms* u, uint32_t* brick_edge,
                             uint32_t* chunk, float* best_ms) {
    if (!ps) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_splat_autotune needs a particle system.");
    GG_CHECK(check_splat(ps, vol, u, "gg_splat_autotune"));
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    static const uint32_t kShapes[][2] = {{0, 0},     {4, 1024},  {4, 4096},  {8, 1024},   {8, 2048},
                                          {8, 4096},  {8, 8192},  {16, 2048}, {16, 4096},  {16, 8192},
                                          {16, 16384}};
    cudaEvent_t e0, e1;
    GG_CUDA(cudaEventCreate(&e0), "autotune events");
    GG_CUDA(cudaEventCreate(&e1), "autotune events");
    float best = 1e30f;
    uint32_t best_edge = 0, best_chunk = 0;
    int status = GG_OK;
    for (const auto& shape : kShapes) {
        if (check_shape(vol, shape[0], shape[1]) != GG_OK) continue;
        float total = 0.0f;
        for (int rep = 0; rep < 4 && status == GG_OK; ++rep) {
            status = gg_volume_clear(vol);
            if (status == GG_OK) status = gg::cuda_status(cudaEventRecord(e0, ctx->stream), "autotune");
            if (status == GG_OK) status = splat_bin_shaped(ps, vol, u, shape[0], shape[1]);
            if (status == GG_OK) status = gg::cuda_status(cudaEventRecord(e1, ctx->stream), "autotune");
            if (status == GG_OK) status = gg::cuda_status(cudaEventSynchronize(e1), "autotune");
            float ms = 0.0f;
            if (status == GG_OK) status = gg::cuda_status(cudaEventElapsedTime(&ms, e0, e1), "autotune");
            if (rep > 0) total += ms;  // the first run also grows the scratch
        }
        if (status != GG_OK) break;
        if (total / 3.0f < best) {
            best = total / 3.0f;
            best_edge = shape[0];
            best_chunk = shape[1];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    GG_CHECK(status);
    GG_CHECK(gg_volume_clear(vol));
    const int mode = u->exactDeposit ? 1 : 0;
    vol->brick_edge[mode] = best_edge;
    vol->brick_chunk[mode] = best_chunk;
    if (brick_edge) *brick_edge = best_edge;
    if (chunk) *chunk = best_chunk;
    if (best_ms) *best_ms = best;
    return GG_OK;
}

GG_API int gg_splat_resolve(gg_volume* vol, const SplatUniforms* u, const gg_particles* ps) {
    GG_CHECK(check_splat(ps, vol, u, "gg_splat_resolve"));
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    ResolveArgs a{vol->sums, vol->emission_surf, vol->velocity_surf, ctx->blackbody, *u,
                  gg_log_d((double)BLACKBODY_T_MIN), gg_log_d((double)BLACKBODY_T_MAX), 0u};
    const uint32_t n = vol->size;
    resolve_kernel<<<dim3((n + 31u) / 32u, (n + kResolveRows - 1u) / kResolveRows, n), dim3(32, kResolveRows), 0,
                     ctx->stream>>>(a);
    return gg::launch_status("splat resolve");
}

GG_API int gg_splat(gg_particles* ps, gg_volume* vol, const SplatUniforms* u) {
    gg::Range range("gg_splat");
    GG_CHECK(gg_splat_bin(ps, vol, u));
    return gg_splat_resolve(vol, u, ps);
}

GG_API int gg_volume_clear(gg_volume* vol) {
    if (!vol) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_clear needs a volume.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t bytes = (uint64_t)vol->size * vol->size * vol->size * 24u;
    const uint64_t n16 = bytes / 16u;  // 24 n^3 is a multiple of 16 for even n; the tail is cleared below
    if (n16) clear_kernel<<<(unsigned)((n16 + 255u) / 256u), 256, 0, ctx->stream>>>(reinterpret_cast<uint4*>(vol->sums), n16);
    GG_CHECK(gg::launch_status("volume clear"));
    if (bytes % 16u) GG_CUDA(cudaMemsetAsync(reinterpret_cast<char*>(vol->sums) + n16 * 16u, 0, bytes % 16u, ctx->stream), "volume clear");
    return GG_OK;
}

GG_API int gg_volume_read_sums(gg_volume* vol, uint32_t* emission, int32_t* momentum, uint32_t* mass) {
    if (!vol || !emission || !momentum || !mass)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_read_sums needs a volume and three output arrays.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t voxels = (uint64_t)vol->size * vol->size * vol->size;
    std::vector<uint32_t> rec(voxels * 6u);
    GG_CUDA(cudaMemcpyAsync(rec.data(), vol->sums, voxels * 24u, cudaMemcpyDeviceToHost, ctx->stream), "sums readback");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "sums readback");
    for (uint64_t i = 0; i < voxels; ++i) {
        emission[2 * i + 0] = rec[6 * i + 0];
        emission[2 * i + 1] = rec[6 * i + 1];
        momentum[3 * i + 0] = (int32_t)rec[6 * i + 2];
        momentum[3 * i + 1] = (int32_t)rec[6 * i + 3];
        momentum[3 * i + 2] = (int32_t)rec[6 * i + 4];
        mass[i] = rec[6 * i + 5];
    }
    return GG_OK;
}

GG_API int gg_volume_write_sums(gg_volume* vol, const uint32_t* emission, const int32_t* momentum, const uint32_t* mass) {
    if (!vol || !emission || !momentum || !mass)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_write_sums needs a volume and three input arrays.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    const uint64_t voxels = (uint64_t)vol->size * vol->size * vol->size;
    std::vector<uint32_t> rec(voxels * 6u);
    for (uint64_t i = 0; i < voxels; ++i) {
        rec[6 * i + 0] = emission[2 * i + 0];
        rec[6 * i + 1] = emission[2 * i + 1];
        rec[6 * i + 2] = (uint32_t)momentum[3 * i + 0];
        rec[6 * i + 3] = (uint32_t)momentum[3 * i + 1];
        rec[6 * i + 4] = (uint32_t)momentum[3 * i + 2];
        rec[6 * i + 5] = mass[i];
    }
    GG_CUDA(cudaMemcpyAsync(vol->sums, rec.data(), voxels * 24u, cudaMemcpyHostToDevice, ctx->stream), "sums upload");
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "sums upload");
    return GG_OK;
}

GG_API int gg_volume_sums(gg_volume* vol, void** device_words, uint64_t* words) {
    if (!vol || !device_words || !words)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_sums needs a volume and two outputs.");
    *device_words = vol->sums;
    *words = (uint64_t)vol->size * vol->size * vol->size * 6u;
    return GG_OK;
}

GG_API int gg_volume_ipc_handle(gg_volume* vol, void* handle) {
    if (!vol || !handle) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_ipc_handle needs a volume and an output.");
    static_assert(sizeof(cudaIpcMemHandle_t) == GG_IPC_HANDLE_BYTES, "the handle size the header states");
    std::lock_guard<std::recursive_mutex> lock(vol->ctx->mu);
    GG_CUDA(cudaSetDevice(vol->ctx->device), "cudaSetDevice");
    cudaIpcMemHandle_t h;
    GG_CUDA(cudaIpcGetMemHandle(&h, vol->sums), "volume sums IPC handle");
    std::memcpy(handle, &h, sizeof h);
    return GG_OK;
}

GG_API int gg_volume_attach_peers(gg_volume* vol, const void* handles, uint32_t count) {
    if (!vol || (count && !handles))
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_attach_peers needs a volume and the handles.");
    if (count > GG_MAX_PEERS)
        return gg::fail(GG_ERR_INVALID_ARGUMENT, "%u peers is more than the %d a volume attaches.", count,
                        GG_MAX_PEERS);
    std::lock_guard<std::recursive_mutex> lock(vol->ctx->mu);
    GG_CUDA(cudaSetDevice(vol->ctx->device), "cudaSetDevice");
    GG_CUDA(cudaStreamSynchronize(vol->ctx->stream), "peer detach");  // no deposit still adds into them
    close_peers(vol);
    for (uint32_t k = 0; k < count; ++k) {
        cudaIpcMemHandle_t h;
        std::memcpy(&h, static_cast<const char*>(handles) + (size_t)k * GG_IPC_HANDLE_BYTES, sizeof h);
        void* p = nullptr;
        const cudaError_t e = cudaIpcOpenMemHandle(&p, h, cudaIpcMemLazyEnablePeerAccess);
        if (e != cudaSuccess) {
            cudaGetLastError();
            close_peers(vol);
            return gg::fail(GG_ERR_DEVICE, "Peer %u's sums could not be opened (%s).", k, cudaGetErrorString(e));
        }
        vol->peer_sums[vol->peers++] = static_cast<uint32_t*>(p);
    }
    return GG_OK;
}

static int copy_volume_array(gg_volume* vol, cudaArray_t arr, void* host, bool to_host) {
    cudaMemcpy3DParms p{};
    cudaExtent e = make_cudaExtent(vol->size, vol->size, vol->size);
    p.extent = e;
    if (to_host) {
        p.srcArray = arr;
        p.dstPtr = make_cudaPitchedPtr(host, vol->size * 8u, vol->size, vol->size);
        p.kind = cudaMemcpyDeviceToHost;
    } else {
        p.dstArray = arr;
        p.srcPtr = make_cudaPitchedPtr(host, vol->size * 8u, vol->size, vol->size);
        p.kind = cudaMemcpyHostToDevice;
    }
    GG_CUDA(cudaMemcpy3DAsync(&p, vol->ctx->stream), "volume copy");
    return GG_OK;
}

GG_API int gg_volume_read(gg_volume* vol, uint16_t* emission_half4, uint16_t* velocity_half4) {
    if (!vol) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_read needs a volume.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (emission_half4) GG_CHECK(copy_volume_array(vol, vol->emission, emission_half4, true));
    if (velocity_half4) GG_CHECK(copy_volume_array(vol, vol->velocity, velocity_half4, true));
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "volume readback");
    return GG_OK;
}

GG_API int gg_volume_write(gg_volume* vol, const uint16_t* emission_half4, const uint16_t* velocity_half4) {
    if (!vol) return gg::fail(GG_ERR_INVALID_ARGUMENT, "gg_volume_write needs a volume.");
    gg_context* ctx = vol->ctx;
    std::lock_guard<std::recursive_mutex> lock(ctx->mu);
    GG_CUDA(cudaSetDevice(ctx->device), "cudaSetDevice");
    if (emission_half4) GG_CHECK(copy_volume_array(vol, vol->emission, const_cast<uint16_t*>(emission_half4), false));
    if (velocity_half4) GG_CHECK(copy_volume_array(vol, vol->velocity, const_cast<uint16_t*>(velocity_half4), false));
    GG_CUDA(cudaStreamSynchronize(ctx->stream), "volume upload");
    return GG_OK;
}

}  // extern "C"
