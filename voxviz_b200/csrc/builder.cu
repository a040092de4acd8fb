// builder.cu - the terrain octree built on the GPU: the fBm heightfield, the
// column-run mip pyramid and the node classification.
//
// The reference builds its octree on the host (GigaVoxelsOctTree::build,
// GigaVoxelsOctTree.cpp:1656-1701): a dense mip pyramid by 2x2x2 box
// averages (GenerateMipMap / GetBoxFilterAverage, :809-960) and a node type
// per node from its brick region (Node::computeNodeType, :1490-1609); its
// offline voxelizer runs the same steps as CUDA kernels (ComputeVoxelMipMap8,
// VoxelizerKernels.cu:1520; ComputeOctTreeNodeType, :2216).  Here every step
// is a kernel over the column-run representation of terrain.h:
//
//   heights_kernel      the solid count of every leaf column (fbm_height)
//   level_count_kernel  per column of mip level m: the run of explicit
//                       voxels between the pure-solid part and the air, from
//                       the four columns below (round-half-up box averages)
//   level_write_kernel  the run's voxels, at offsets from a scan of the counts
//   classify_kernel     per node of tree level d: constant or not and its
//                       value (the region with its 1-voxel border, the edge
//                       rule and the transparent-match rule)
//   child_write_kernel  the next level's nodes: 8 children of every node that
//                       has children, at offsets from a scan
//
// The host then numbers the blocks depth first (GigaVoxelsOctTree::
// from_levels) and keeps a copy of the pyramid for host-side checks.  Every
// value equals the host build's (float arithmetic without contraction).
#include <cuda_runtime.h>

#include <memory>
#include <string>
#include <vector>

#include "octree.h"
#include "terrain.h"

namespace vv {

namespace {

// ---- fBm heightfield (terrain.cpp's arithmetic, on the device) ----------

__device__ __forceinline__ uint32_t lattice_hash_d(uint32_t x, uint32_t y, uint32_t seed) {
    uint32_t h = seed * 0x9E3779B9u;
    h ^= x * 0x85EBCA6Bu;
    h = (h << 13) | (h >> 19);
    h ^= y * 0xC2B2AE35u;
    h ^= h >> 16;
    h *= 0x7FEB352Du;
    h ^= h >> 15;
    h *= 0x846CA68Bu;
    h ^= h >> 16;
    return h;
}

__device__ __forceinline__ float lattice_value_d(int32_t x, int32_t y, uint32_t seed) {
    return (float)(lattice_hash_d((uint32_t)x, (uint32_t)y, seed) >> 8) * (1.0f / 16777216.0f);
}

__device__ __forceinline__ float smoothstep01_d(float t) { return (t * t) * (3.0f - 2.0f * t); }

__device__ float value_noise_d(float x, float y, uint32_t seed) {
    const float fx = floorf(x), fy = floorf(y);
    const int32_t ix = (int32_t)fx, iy = (int32_t)fy;
    const float sx = smoothstep01_d(x - fx), sy = smoothstep01_d(y - fy);
    const float v00 = lattice_value_d(ix, iy, seed);
    const float v10 = lattice_value_d(ix + 1, iy, seed);
    const float v01 = lattice_value_d(ix, iy + 1, seed);
    const float v11 = lattice_value_d(ix + 1, iy + 1, seed);
    const float a = v00 + (v10 - v00) * sx;
    const float b = v01 + (v11 - v01) * sx;
    return a + (b - a) * sy;
}

struct FbmParams {
    uint32_t seed;
    int octaves;
    float lacunarity, gain;
    int base_cells;
};

__device__ float fbm_height_d(const FbmParams& p, float u, float v) {
    float sum = 0.0f, amp = 1.0f, norm = 0.0f, freq = (float)p.base_cells;
    for (int o = 0; o < p.octaves; ++o) {
        const uint32_t s = p.seed + (uint32_t)o * 0x632BE5ABu;
        sum = sum + amp * value_noise_d(u * freq, v * freq, s);
        norm = norm + amp;
        amp = amp * p.gain;
        freq = freq * p.lacunarity;
    }
    return sum / norm;
}

__global__ void heights_kernel(FbmParams p, int n, int32_t* __restrict__ heights, uint16_t* __restrict__ s0) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= n) return;
    const float inv = 1.0f / (float)n;
    const float h = fbm_height_d(p, (float)x * inv, (float)y * inv);
    const float t = h * (float)n;
    int H = (int)ceilf(t);
    if (H < 0) H = 0;
    if (H > n) H = n;
    heights[(size_t)y * n + x] = H;
    s0[(size_t)y * n + x] = (uint16_t)H;
}

// ---- the column-run pyramid ----------------------------------------------

__constant__ uint32_t c_band[8];

struct Level {
    int dim;
    const uint16_t* s;
    const uint16_t* r;     // nullptr at level 0
    const uint32_t* off;   // nullptr at level 0
    const uint32_t* data;  // nullptr at level 0
};

// RGBA8 voxel (x,y,z) of mip level m (terrain.h TerrainVolume::voxel).
__device__ __forceinline__ uint32_t voxel_d(const Level& L, int m, int depth, int x, int y, int z) {
    const size_t c = (size_t)y * L.dim + x;
    const int s = L.s[c];
    if (z < s) return c_band[((z << m) >> depth) & 7];
    if (L.r) {
        const int r = L.r[c];
        if (z < s + r) return L.data[L.off[c] + (uint32_t)(z - s)];
    }
    return 0u;
}

// Voxel Z of column (X,Y) of level m: the 2x2x2 box average of level m-1
// with GetBoxFilterAverage's rounding, floor(sum / 8 + 0.5) = (sum + 4) >> 3.
__device__ __forceinline__ uint32_t box_voxel(const Level& P, int m, int depth, int X, int Y, int Z) {
    uint32_t sr = 0, sg = 0, sb = 0, sa = 0;
#pragma unroll
    for (int k = 0; k < 2; ++k)
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i) {
                const uint32_t v = voxel_d(P, m - 1, depth, 2 * X + i, 2 * Y + j, 2 * Z + k);
                sr += v & 255u;
                sg += (v >> 8) & 255u;
                sb += (v >> 16) & 255u;
                sa += v >> 24;
            }
    return ((sr + 4) >> 3) | (((sg + 4) >> 3) << 8) | (((sb + 4) >> 3) << 16) | (((sa + 4) >> 3) << 24);
}

__device__ __forceinline__ uint32_t band_of(int m, int depth, int z) { return c_band[((z << m) >> depth) & 7]; }

// The explicit run of column (X,Y) of level m: voxels of [zlo, zhi) (the
// span of the four columns below) minus a leading part equal to the band
// colour the pure-solid rule gives and a trailing part of transparent black.
__device__ __forceinline__ void column_run(const Level& P, int m, int depth, int X, int Y, int& zs, int& len) {
    const int dp = P.dim;
    int lo = 1 << 30, hi = 0;
#pragma unroll
    for (int j = 0; j < 2; ++j)
#pragma unroll
        for (int i = 0; i < 2; ++i) {
            const size_t c = (size_t)(2 * Y + j) * dp + (2 * X + i);
            const int s = P.s[c], e = s + (P.r ? (int)P.r[c] : 0);
            lo = min(lo, s);
            hi = max(hi, e);
        }
    const int zlo = lo >> 1, zhi = (hi + 1) >> 1;
    int b = zlo;
    while (b < zhi && box_voxel(P, m, depth, X, Y, b) == band_of(m, depth, b)) ++b;
    int e = zhi;
    while (e > b && box_voxel(P, m, depth, X, Y, e - 1) == 0u) --e;
    zs = b;
    len = e - b;
}

__global__ void level_count_kernel(Level P, int m, int depth, int d, uint16_t* __restrict__ s,
                                   uint16_t* __restrict__ r, uint32_t* __restrict__ len) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y;
    if (X >= d) return;
    int zs, n;
    column_run(P, m, depth, X, Y, zs, n);
    const size_t c = (size_t)Y * d + X;
    s[c] = (uint16_t)zs;
    r[c] = (uint16_t)n;
    len[c] = (uint32_t)n;
}

__global__ void level_write_kernel(Level P, int m, int depth, int d, const uint16_t* __restrict__ s,
                                   const uint16_t* __restrict__ r, const uint32_t* __restrict__ off,
                                   uint32_t* __restrict__ data) {
    const int X = blockIdx.x * blockDim.x + threadIdx.x, Y = blockIdx.y;
    if (X >= d) return;
    const size_t c = (size_t)Y * d + X;
    const int zs = s[c], n = r[c];
    uint32_t* out = data + off[c];
    for (int q = 0; q < n; ++q) out[q] = box_voxel(P, m, depth, X, Y, zs + q);
}

// ---- exclusive scan of uint32 (blocks of 1024, block sums scanned in turn) -

constexpr int kScanBlock = 1024;

__global__ void scan_blocks_kernel(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, size_t n,
                                   uint32_t* __restrict__ sums) {
    __shared__ uint32_t warp_tot[32];
    const size_t i = (size_t)blockIdx.x * kScanBlock + threadIdx.x;
    const uint32_t v = i < n ? in[i] : 0u;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    if (w == 0) {
        uint32_t t = warp_tot[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, t, o);
            if (lane >= o) t += y;
        }
        warp_tot[lane] = t;  // inclusive over warps
    }
    __syncthreads();
    const uint32_t before = w ? warp_tot[w - 1] : 0u;
    if (i < n) out[i] = before + x - v;
    if (threadIdx.x == kScanBlock - 1) sums[blockIdx.x] = warp_tot[31];
}

__global__ void scan_add_kernel(uint32_t* __restrict__ out, size_t n, const uint32_t* __restrict__ sums) {
    const size_t i = (size_t)blockIdx.x * kScanBlock + threadIdx.x;
    if (i < n && blockIdx.x > 0) out[i] += sums[blockIdx.x];
}

// out = exclusive scan of in (n values); returns the total in *total (host).
cudaError_t exclusive_scan(const uint32_t* in, uint32_t* out, size_t n, uint64_t* total, cudaStream_t st) {
    if (n == 0) {
        *total = 0;
        return cudaSuccess;
    }
    const size_t blocks = (n + kScanBlock - 1) / kScanBlock;
    uint32_t* sums = nullptr;
    uint32_t* sums_scan = nullptr;
    cudaError_t e = cudaMalloc(&sums, blocks * 4);
    if (e == cudaSuccess) e = cudaMalloc(&sums_scan, blocks * 4);
    if (e == cudaSuccess) {
        scan_blocks_kernel<<<(unsigned)blocks, kScanBlock, 0, st>>>(in, out, n, sums);
        e = cudaGetLastError();
    }
    if (blocks == 1) {  // one block: its sum is the total
        uint32_t t = 0;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&t, sums, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e == cudaSuccess) *total = t;
    } else {
        uint64_t sub_total = 0;
        if (e == cudaSuccess) e = exclusive_scan(sums, sums_scan, blocks, &sub_total, st);
        if (e == cudaSuccess) {
            scan_add_kernel<<<(unsigned)blocks, kScanBlock, 0, st>>>(out, n, sums_scan);
            e = cudaGetLastError();
        }
        if (e == cudaSuccess) *total = sub_total;
    }
    if (sums) cudaFree(sums);
    if (sums_scan) cudaFree(sums_scan);
    return e;
}

// ---- node classification ---------------------------------------------------

// Node::computeNodeType for node (i,j,k) of tree level d = L - m
// (classify_node in octree.cpp): the 8^3 voxels of mip level m plus a
// 1-voxel border inside the level; a region touching the volume edge is
// compared against transparent black; transparent voxels match any
// transparent value.
__device__ bool classify_d(const Level& M, int m, int depth, int i, int j, int k, uint32_t& cval) {
    const int dim = M.dim;
    const int idx[3] = {i, j, k};
    int a0[3], a1[3];
    bool edge = false;
#pragma unroll
    for (int ax = 0; ax < 3; ++ax) {
        a0[ax] = 8 * idx[ax];
        a1[ax] = a0[ax] + 8;
        if (a0[ax] != 0) a0[ax] -= 1;
        if (a1[ax] <= dim - 1) a1[ax] += 1;
        if (a1[ax] > dim) a1[ax] = dim;
        if (a0[ax] == 0 || a1[ax] == dim) edge = true;
    }
    const uint32_t cv = edge ? 0u : voxel_d(M, m, depth, a0[0], a0[1], a0[2]);
    int minS = 1 << 30, maxE = 0;
    for (int y = a0[1]; y < a1[1]; ++y)
        for (int x = a0[0]; x < a1[0]; ++x) {
            const size_t c = (size_t)y * dim + x;
            const int s = M.s[c];
            minS = min(minS, s);
            maxE = max(maxE, s + (M.r ? (int)M.r[c] : 0));
        }
    if (a0[2] >= maxE) {  // every voxel transparent black
        cval = cv;
        return true;
    }
    if (a1[2] <= minS) {  // every voxel pure solid, colour by band
        if (edge) return false;
        if (((a0[2] << m) >> depth & 7) != (((a1[2] - 1) << m) >> depth & 7)) return false;
        cval = cv;
        return true;
    }
    const bool cv_clear = (cv >> 24) == 0u;
    for (int z = a0[2]; z < a1[2]; ++z)
        for (int y = a0[1]; y < a1[1]; ++y)
            for (int x = a0[0]; x < a1[0]; ++x) {
                const uint32_t v = voxel_d(M, m, depth, x, y, z);
                if ((v >> 24) == 0u && cv_clear) continue;
                if (v != cv) return false;
            }
    cval = cv;
    return true;
}

__global__ void classify_kernel(Level M, int m, int depth, size_t n, const uint16_t* __restrict__ ni,
                                const uint16_t* __restrict__ nj, const uint16_t* __restrict__ nk,
                                uint8_t* __restrict__ isc, uint32_t* __restrict__ cval, int collapse,
                                uint32_t* __restrict__ children) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    uint32_t cv = 0u;
    const bool c = classify_d(M, m, depth, ni[q], nj[q], nk[q], cv);
    isc[q] = c ? 1 : 0;
    cval[q] = c ? cv : 0u;
    if (children) children[q] = (collapse && c) ? 0u : 8u;
}

__global__ void child_write_kernel(size_t n, const uint16_t* __restrict__ ni, const uint16_t* __restrict__ nj,
                                   const uint16_t* __restrict__ nk, const uint32_t* __restrict__ children,
                                   const uint32_t* __restrict__ off, uint16_t* __restrict__ ci,
                                   uint16_t* __restrict__ cj, uint16_t* __restrict__ ck,
                                   uint32_t* __restrict__ parent) {
    const size_t q = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n || children[q] == 0u) return;
    const uint32_t o = off[q];
    for (int c = 0; c < 8; ++c) {
        ci[o + c] = (uint16_t)(2 * ni[q] + (c & 1));
        cj[o + c] = (uint16_t)(2 * nj[q] + ((c >> 1) & 1));
        ck[o + c] = (uint16_t)(2 * nk[q] + (c >> 2));
        parent[o + c] = (uint32_t)q;
    }
}

// Device allocations freed at scope exit.
struct DevBufs {
    std::vector<void*> p;
    ~DevBufs() {
        for (void* q : p) cudaFree(q);
    }
    template <class T>
    cudaError_t alloc(T** out, size_t count) {
        void* q = nullptr;
        cudaError_t e = cudaMalloc(&q, count ? count * sizeof(T) : sizeof(T));
        if (e != cudaSuccess) return e;
        p.push_back(q);
        *out = (T*)q;
        return cudaSuccess;
    }
};

template <class T>
cudaError_t download(std::vector<T>& v, const T* d, size_t n) {
    v.resize(n);
    return n ? cudaMemcpy(v.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost) : cudaSuccess;
}

}  // namespace

// The terrain volume and the classified tree levels of GigaVoxelsOctTree::
// build, computed on the current CUDA device.  Returns an error message, or
// an empty string.
std::string gpu_build_terrain(const TerrainParams& p, bool collapse, std::shared_ptr<TerrainVolume>& vol_out,
                              std::vector<TreeLevel>& levels) {
    if (p.depth < 0 || p.depth > 10) return "terrain depth must be in [0,10]";
    const int L = p.depth, n0 = 8 << L;
    cudaStream_t st = 0;
    DevBufs bufs;
    std::vector<MipLevel> mips((size_t)L + 1);
    std::vector<Level> dl((size_t)L + 1);
    uint32_t band[8];
    for (int b = 0; b < 8; ++b) band[b] = band_colour(b);
    cudaError_t e = cudaMemcpyToSymbol(c_band, band, sizeof(band));
    // heights and level 0
    int32_t* d_h = nullptr;
    uint16_t* d_s0 = nullptr;
    if (e == cudaSuccess) e = bufs.alloc(&d_h, (size_t)n0 * n0);
    if (e == cudaSuccess) e = bufs.alloc(&d_s0, (size_t)n0 * n0);
    if (e == cudaSuccess) {
        FbmParams fp{p.seed, p.octaves, p.lacunarity, p.gain, p.base_cells};
        heights_kernel<<<dim3((unsigned)((n0 + 255) / 256), (unsigned)n0), 256, 0, st>>>(fp, n0, d_h, d_s0);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) return std::string("heights: ") + cudaGetErrorString(e);
    dl[0] = Level{n0, d_s0, nullptr, nullptr, nullptr};
    // levels 1..L
    for (int m = 1; m <= L && e == cudaSuccess; ++m) {
        const int d = n0 >> m;
        const size_t cols = (size_t)d * d;
        uint16_t *s = nullptr, *r = nullptr;
        uint32_t *len = nullptr, *off = nullptr, *data = nullptr;
        e = bufs.alloc(&s, cols);
        if (e == cudaSuccess) e = bufs.alloc(&r, cols);
        if (e == cudaSuccess) e = bufs.alloc(&len, cols);
        if (e == cudaSuccess) e = bufs.alloc(&off, cols);
        if (e != cudaSuccess) break;
        const dim3 grid((unsigned)((d + 127) / 128), (unsigned)d);
        level_count_kernel<<<grid, 128, 0, st>>>(dl[(size_t)m - 1], m, L, d, s, r, len);
        e = cudaGetLastError();
        uint64_t total = 0;
        if (e == cudaSuccess) e = exclusive_scan(len, off, cols, &total, st);
        if (e == cudaSuccess && total > 0xFFFFFFFFull) return "mip level too large for 32-bit offsets";
        if (e == cudaSuccess) e = bufs.alloc(&data, (size_t)total);
        if (e == cudaSuccess) {
            level_write_kernel<<<grid, 128, 0, st>>>(dl[(size_t)m - 1], m, L, d, s, r, off, data);
            e = cudaGetLastError();
        }
        dl[(size_t)m] = Level{d, s, r, off, data};
        if (e == cudaSuccess) {
            MipLevel& H = mips[(size_t)m];
            H.dim = d;
            std::vector<uint32_t> off32;
            e = download(H.s, s, cols);
            if (e == cudaSuccess) e = download(H.r, r, cols);
            if (e == cudaSuccess) e = download(off32, off, cols);
            if (e == cudaSuccess) e = download(H.data, data, (size_t)total);
            H.off.assign(off32.begin(), off32.end());
        }
    }
    if (e != cudaSuccess) return std::string("mip pyramid: ") + cudaGetErrorString(e);
    std::vector<int32_t> heights;
    {
        MipLevel& H0 = mips[0];
        H0.dim = n0;
        e = download(heights, d_h, (size_t)n0 * n0);
        if (e == cudaSuccess) e = download(H0.s, d_s0, (size_t)n0 * n0);
        H0.r.assign((size_t)n0 * n0, 0);
        H0.off.assign((size_t)n0 * n0, 0);
    }
    if (e != cudaSuccess) return std::string("heights download: ") + cudaGetErrorString(e);
    // tree levels: the root, then the children of every node with children
    levels.assign((size_t)L + 1, TreeLevel());
    size_t n = 1;
    uint16_t *ni = nullptr, *nj = nullptr, *nk = nullptr;
    uint32_t* npar = nullptr;
    e = bufs.alloc(&ni, 1);
    if (e == cudaSuccess) e = bufs.alloc(&nj, 1);
    if (e == cudaSuccess) e = bufs.alloc(&nk, 1);
    if (e == cudaSuccess) e = bufs.alloc(&npar, 1);
    const uint16_t zero16 = 0;
    const uint32_t noparent = kNoParent;
    if (e == cudaSuccess) e = cudaMemcpy(ni, &zero16, 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(nj, &zero16, 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(nk, &zero16, 2, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(npar, &noparent, 4, cudaMemcpyHostToDevice);
    for (int d = 0; d <= L && e == cudaSuccess; ++d) {
        const int m = L - d;
        uint8_t* isc = nullptr;
        uint32_t *cval = nullptr, *children = nullptr, *coff = nullptr;
        e = bufs.alloc(&isc, n);
        if (e == cudaSuccess) e = bufs.alloc(&cval, n);
        if (e == cudaSuccess && d < L) e = bufs.alloc(&children, n);
        if (e == cudaSuccess && d < L) e = bufs.alloc(&coff, n);
        if (e != cudaSuccess) break;
        classify_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(dl[(size_t)m], m, L, n, ni, nj, nk, isc, cval,
                                                                      collapse ? 1 : 0, children);
        e = cudaGetLastError();
        TreeLevel& T = levels[(size_t)d];
        if (e == cudaSuccess) e = download(T.i, (const uint16_t*)ni, n);
        if (e == cudaSuccess) e = download(T.j, (const uint16_t*)nj, n);
        if (e == cudaSuccess) e = download(T.k, (const uint16_t*)nk, n);
        if (e == cudaSuccess) e = download(T.parent, (const uint32_t*)npar, n);
        if (e == cudaSuccess) e = download(T.isc, (const uint8_t*)isc, n);
        if (e == cudaSuccess) e = download(T.cval, (const uint32_t*)cval, n);
        if (e != cudaSuccess || d == L) break;
        uint64_t next = 0;
        e = exclusive_scan(children, coff, n, &next, st);
        if (e != cudaSuccess) break;
        if (next > 0xFFFFFFFFull) return "tree level too large";
        uint16_t *ci = nullptr, *cj = nullptr, *ck = nullptr;
        uint32_t* cpar = nullptr;
        e = bufs.alloc(&ci, (size_t)next);
        if (e == cudaSuccess) e = bufs.alloc(&cj, (size_t)next);
        if (e == cudaSuccess) e = bufs.alloc(&ck, (size_t)next);
        if (e == cudaSuccess) e = bufs.alloc(&cpar, (size_t)next);
        if (e != cudaSuccess) break;
        child_write_kernel<<<(unsigned)((n + 127) / 128), 128, 0, st>>>(n, ni, nj, nk, children, coff, ci, cj, ck,
                                                                         cpar);
        e = cudaGetLastError();
        ni = ci;
        nj = cj;
        nk = ck;
        npar = cpar;
        n = (size_t)next;
    }
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) return std::string("classification: ") + cudaGetErrorString(e);
    vol_out = std::make_shared<TerrainVolume>(p, std::move(heights), std::move(mips));
    return std::string();
}

}  // namespace vv
