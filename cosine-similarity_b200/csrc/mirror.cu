// Lower triangle of a symmetric dense result from its upper triangle.
//
// matchms' is_symmetric=True scores only the pairs (i, j) with i <= j and
// gives (j, i) the same result.  The kernels write the upper triangle; this
// kernel copies it down.  Work unit: a tile (ti, tj) with tj <= ti of the
// lower triangle; its source tile (tj, ti) is read row-wise into shared
// memory and written back transposed, so reads and writes are both coalesced.
// Pure copy: 2 x (4 + 4 + 1) bytes per lower-triangle pair of HBM traffic.
// When the row stride and the three base pointers are 16-byte aligned the
// tiles are 64 x 64 and every global access is a 16-byte vector (nine per
// thread in flight per tile); otherwise 32 x 32 tiles with scalar accesses.
#include <algorithm>
#include <cmath>
#include <cstdint>

#include "cms_internal.cuh"

namespace cms {
namespace {

constexpr int kTile = 32;
constexpr int kThreads = 256;  // 32 x 8
constexpr int kVTile = 64;

// tile index t -> (ti, tj) with t = ti * (ti + 1) / 2 + tj, 0 <= tj <= ti
__device__ __forceinline__ void lower_tile(int64_t t, int64_t& ti, int64_t& tj) {
    ti = (int64_t)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
    while (ti > 0 && ti * (ti + 1) / 2 > t) --ti;
    while ((ti + 1) * (ti + 2) / 2 <= t) ++ti;
    tj = t - ti * (ti + 1) / 2;
}

// 64 x 64 tiles, 16-byte accesses; needs ld % 16 == 0 and 16-byte aligned
// score / matches / overflow (matches and overflow may be null)
__global__ void __launch_bounds__(kThreads) mirror_vec_kernel(DenseOut d, int64_t n,
                                                              const uint32_t* bad) {
    if (bad && *bad) return;
    __shared__ float s_sc[kVTile][kVTile + 1];
    __shared__ int32_t s_mt[kVTile][kVTile + 1];
    __shared__ uint8_t s_of[kVTile][kVTile + 4];
    const int64_t T = (n + kVTile - 1) / kVTile;
    const int64_t n_tiles = T * (T + 1) / 2;
    const int tid = threadIdx.x;
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        int64_t ti, tj;
        lower_tile(t, ti, tj);
        const int64_t r0 = ti * kVTile, c0 = tj * kVTile;
        __syncthreads();
        // source rows c0 + yy, columns r0 + 4 * c4 .. + 3 (f32 / i32)
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int e = tid + kThreads * k;
            const int yy = e >> 4, c4 = e & 15;
            const int64_t sr = c0 + yy, sc = r0 + 4 * c4;
            if (sr >= n || sc >= n) continue;
            const int64_t o = sr * d.ld + sc;
            float4 v;
            if (sc + 3 < n) {
                v = __ldcs(reinterpret_cast<const float4*>(d.score + o));
            } else {
                v = make_float4(d.score[o], sc + 1 < n ? d.score[o + 1] : 0.f,
                                sc + 2 < n ? d.score[o + 2] : 0.f, 0.f);
            }
            s_sc[yy][4 * c4] = v.x;
            s_sc[yy][4 * c4 + 1] = v.y;
            s_sc[yy][4 * c4 + 2] = v.z;
            s_sc[yy][4 * c4 + 3] = v.w;
            if (d.matches) {
                int4 m;
                if (sc + 3 < n) {
                    m = __ldcs(reinterpret_cast<const int4*>(d.matches + o));
                } else {
                    m = make_int4(d.matches[o], sc + 1 < n ? d.matches[o + 1] : 0,
                                  sc + 2 < n ? d.matches[o + 2] : 0, 0);
                }
                s_mt[yy][4 * c4] = m.x;
                s_mt[yy][4 * c4 + 1] = m.y;
                s_mt[yy][4 * c4 + 2] = m.z;
                s_mt[yy][4 * c4 + 3] = m.w;
            }
        }
        if (d.overflow) {
            // source rows c0 + yy, columns r0 + 16 * c .. + 15 (u8)
            const int yy = tid >> 2, c = tid & 3;
            const int64_t sr = c0 + yy, sc = r0 + 16 * c;
            if (sr < n && sc < n) {
                const int64_t o = sr * d.ld + sc;
                uint4 v;
                if (sc + 15 < n) {
                    v = __ldcs(reinterpret_cast<const uint4*>(d.overflow + o));
                } else {
                    uint32_t w[4] = {0u, 0u, 0u, 0u};
                    for (int b = 0; b < 16 && sc + b < n; ++b)
                        w[b >> 2] |= (uint32_t)d.overflow[o + b] << (8 * (b & 3));
                    v = make_uint4(w[0], w[1], w[2], w[3]);
                }
                uint32_t* dst = reinterpret_cast<uint32_t*>(&s_of[yy][16 * c]);
                dst[0] = v.x;
                dst[1] = v.y;
                dst[2] = v.z;
                dst[3] = v.w;
            }
        }
        __syncthreads();
        // destination rows r0 + yy, columns c0 + 4 * c4 .. + 3, where row > column
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int e = tid + kThreads * k;
            const int yy = e >> 4, c4 = e & 15;
            const int64_t dr = r0 + yy, dc = c0 + 4 * c4;
            if (dr >= n || dc >= dr) continue;
            const int64_t o = dr * d.ld + dc;
            const int sx = 4 * c4;
            if (dc + 3 < dr) {  // dr < n, so all four columns are inside
                __stcs(reinterpret_cast<float4*>(d.score + o),
                       make_float4(s_sc[sx][yy], s_sc[sx + 1][yy], s_sc[sx + 2][yy],
                                   s_sc[sx + 3][yy]));
                if (d.matches)
                    __stcs(reinterpret_cast<int4*>(d.matches + o),
                           make_int4(s_mt[sx][yy], s_mt[sx + 1][yy], s_mt[sx + 2][yy],
                                     s_mt[sx + 3][yy]));
            } else {
                for (int b = 0; b < 4 && dc + b < dr; ++b) {
                    d.score[o + b] = s_sc[sx + b][yy];
                    if (d.matches) d.matches[o + b] = s_mt[sx + b][yy];
                }
            }
        }
        if (d.overflow) {
            const int yy = tid >> 2, c = tid & 3;
            const int64_t dr = r0 + yy, dc = c0 + 16 * c;
            if (dr < n && dc < dr) {
                const int64_t o = dr * d.ld + dc;
                const int sx = 16 * c;
                if (dc + 15 < dr) {
                    uint32_t w[4];
#pragma unroll
                    for (int q = 0; q < 4; ++q)
                        w[q] = (uint32_t)s_of[sx + 4 * q][yy] |
                               ((uint32_t)s_of[sx + 4 * q + 1][yy] << 8) |
                               ((uint32_t)s_of[sx + 4 * q + 2][yy] << 16) |
                               ((uint32_t)s_of[sx + 4 * q + 3][yy] << 24);
                    __stcs(reinterpret_cast<uint4*>(d.overflow + o),
                           make_uint4(w[0], w[1], w[2], w[3]));
                } else {
                    for (int b = 0; b < 16 && dc + b < dr; ++b) d.overflow[o + b] = s_of[sx + b][yy];
                }
            }
        }
    }
}

__global__ void __launch_bounds__(kThreads) mirror_kernel(DenseOut d, int64_t n,
                                                          const uint32_t* bad) {
    if (bad && *bad) return;
    __shared__ float s_sc[kTile][kTile + 1];
    __shared__ int32_t s_mt[kTile][kTile + 1];
    __shared__ uint8_t s_of[kTile][kTile + 4];
    const int64_t T = (n + kTile - 1) / kTile;
    const int64_t n_tiles = T * (T + 1) / 2;
    const int x = threadIdx.x & 31, y = threadIdx.x >> 5;
    for (int64_t t = blockIdx.x; t < n_tiles; t += gridDim.x) {
        int64_t ti, tj;
        lower_tile(t, ti, tj);
        const int64_t r0 = ti * kTile, c0 = tj * kTile;
        __syncthreads();
        // source: rows c0 + yy, columns r0 + x, where row < column
        for (int yy = y; yy < kTile; yy += 8) {
            const int64_t sr = c0 + yy, sc = r0 + x;
            if (sc < n && sr < sc) {
                const int64_t o = sr * d.ld + sc;
                s_sc[yy][x] = d.score[o];
                if (d.matches) s_mt[yy][x] = d.matches[o];
                if (d.overflow) s_of[yy][x] = d.overflow[o];
            }
        }
        __syncthreads();
        // destination: rows r0 + yy, columns c0 + x, where row > column
        for (int yy = y; yy < kTile; yy += 8) {
            const int64_t dr = r0 + yy, dc = c0 + x;
            if (dr < n && dc < dr) {
                const int64_t o = dr * d.ld + dc;
                d.score[o] = s_sc[x][yy];
                if (d.matches) d.matches[o] = s_mt[x][yy];
                if (d.overflow) d.overflow[o] = s_of[x][yy];
            }
        }
    }
}

}  // namespace

int launch_mirror(const DenseOut& d, int64_t n, const uint32_t* bad, int sm_count,
                  cudaStream_t s) {
    if (n < 2) return CMS_OK;
    auto aligned = [](const void* p) { return p == nullptr || ((uintptr_t)p & 15) == 0; };
    const bool vec = d.ld % 16 == 0 && aligned(d.score) && aligned(d.matches) &&
                     aligned(d.overflow);
    const int tile = vec ? kVTile : kTile;
    const int64_t T = (n + tile - 1) / tile;
    const int64_t tiles = T * (T + 1) / 2;
    const int grid = (int)std::max<int64_t>(1, std::min<int64_t>(tiles, (int64_t)sm_count * 8));
    if (vec)
        mirror_vec_kernel<<<grid, kThreads, 0, s>>>(d, n, bad);
    else
        mirror_kernel<<<grid, kThreads, 0, s>>>(d, n, bad);
    CMS_CUDA_TRY(cudaGetLastError());
    return CMS_OK;
}

}  // namespace cms
