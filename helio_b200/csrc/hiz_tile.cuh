// hiz_tile.cuh — one 64x64 tile of the fused Hi-Z build (levels 0..6) and the
// per-view tail (levels 7..), shared by the standalone Hi-Z kernel and the
// persistent multi-view kernel.
//
// Reference: crates/helio-pass-hiz/shaders/hiz_depth_copy.wgsl:13-19 (level 0 copy)
// and hiz_build.wgsl:12-23 (dst = max(1, dim >> (m+1)); the +1 neighbours are
// clamped to src_size - 1, so odd sizes drop the last row / column).
//
//   * a CTA of 256 threads owns a 64x64 tile of level 0: each thread loads a 4x4
//     block with 128-bit loads, reduces it in registers to levels 1 and 2, warp
//     shuffles give level 3, shared memory + warp 0 give levels 4..6;
//   * the warp 0 of the last CTA of a view to finish (atomic ticket after a fence)
//     builds the remaining levels 7.. from level 6.
// Every level-l texel is exactly max() over a rectangle of level 0 (max is exact)
// and each 2x2 step applies the reference's clamp rule (a source dimension of 1
// reuses the same texel), so the result is bit-identical to the per-level chain.
#pragma once

#include "common.cuh"
#include "kernels.h"

namespace helio {

// One 2x2 step of hiz_build.wgsl: a=(2x,2y) b=(2x+1,2y) c=(2x,2y+1) d=(2x+1,2y+1);
// a source dimension of 1 clamps the +1 neighbour back onto the same texel.
__device__ __forceinline__ float hiz_red4(float a, float b, float c, float d, bool xc, bool yc) {
    if (xc) {
        b = a;
        d = c;
    }
    if (yc) {
        c = a;
        d = b;
    }
    return fmaxf(fmaxf(a, b), fmaxf(c, d));
}

constexpr int kHizTailBuf = 2304;  // floats per shared tail buffer

// Levels 7.. of one pyramid, built from level 6 by kWarps warps (warp index w =
// (threadIdx.x >> 5) % kWarps; every thread of those warps calls it). The level loop is
// unrolled so that J's per-level fields are read at fixed offsets, and each level is
// walked by rows: warp w takes rows w, w + kWarps, ... in rounds of kRows rows per lane
// (kRows x 4 loads in flight), lanes take the columns, so no index needs a division.
// Level 7 reads level 6 from global memory (written by other CTAs, through L2); a level
// that fits a shared buffer is kept there for the next level.
template <int kWarps, int kRows>
__device__ __forceinline__ void hiz_tail_sync() {
    if (kWarps == 1) __syncwarp();
    else __syncthreads();
}

template <int kWarps, int kRows>
static __device__ __forceinline__ void hiz_tail_body(const HizJob& J, float* bufA, float* bufB) {
    const uint32_t lane = threadIdx.x & 31u, w = (threadIdx.x >> 5) % (uint32_t)kWarps;
    const uint32_t mips = J.mip_count;
    float* cur = nullptr;  // shared copy of the current source level (or null: read global)
    float* nxt = bufA;
#pragma unroll
    for (int l = 7; l < HELIO_HIZ_MAX_MIPS; ++l) {
        if ((uint32_t)l >= mips) break;
        const uint32_t sw = J.lw[l - 1], sh = J.lh[l - 1], sp = J.lpitch[l - 1];
        const uint32_t dw = J.lw[l], dh = J.lh[l], dp = J.lpitch[l];
        const float* __restrict__ src = J.levels[l - 1];
        float* __restrict__ dst = J.levels[l];
        const bool fits = (size_t)dw * dh <= (size_t)kHizTailBuf;
        for (uint32_t y0 = w; y0 < dh; y0 += (uint32_t)(kWarps * kRows)) {
            for (uint32_t x = lane; x < dw; x += 32u) {
                const uint32_t x0 = 2u * x, x1 = min(x0 + 1u, sw - 1u);
                float q[kRows][4];
#pragma unroll
                for (int r = 0; r < kRows; ++r) {
                    const uint32_t y = y0 + (uint32_t)(kWarps * r);
                    if (y < dh) {
                        const uint32_t ya = 2u * y, yb = min(ya + 1u, sh - 1u);
                        if (cur) {
                            q[r][0] = cur[ya * sw + x0];
                            q[r][1] = cur[ya * sw + x1];
                            q[r][2] = cur[yb * sw + x0];
                            q[r][3] = cur[yb * sw + x1];
                        } else {
                            q[r][0] = __ldcg(src + (size_t)ya * sp + x0);
                            q[r][1] = __ldcg(src + (size_t)ya * sp + x1);
                            q[r][2] = __ldcg(src + (size_t)yb * sp + x0);
                            q[r][3] = __ldcg(src + (size_t)yb * sp + x1);
                        }
                    }
                }
#pragma unroll
                for (int r = 0; r < kRows; ++r) {
                    const uint32_t y = y0 + (uint32_t)(kWarps * r);
                    if (y < dh) {
                        const float v = fmaxf(fmaxf(q[r][0], q[r][1]), fmaxf(q[r][2], q[r][3]));
                        dst[(size_t)y * dp + x] = v;
                        if (fits) nxt[y * dw + x] = v;
                    }
                }
            }
        }
        hiz_tail_sync<kWarps, kRows>();
        if (fits) {
            cur = nxt;
            nxt = (nxt == bufA) ? bufB : bufA;
        } else {
            cur = nullptr;
        }
    }
}

// The same as a call of its own (callers that keep few registers live across it).
template <int kWarps, int kRows>
static __device__ __noinline__ void hiz_tail_in(const HizJob& J, float* bufA, float* bufB) {
    hiz_tail_body<kWarps, kRows>(J, bufA, bufB);
}

// The tail with its two shared buffers declared here (bufA / bufB of kHizTailBuf floats).
template <int kWarps, int kRows>
static __device__ __forceinline__ void hiz_tail(const HizJob& J) {
    __shared__ float bufA[kHizTailBuf];
    __shared__ float bufB[kHizTailBuf];
    hiz_tail_in<kWarps, kRows>(J, bufA, bufB);
}

// The tail by one warp (lane = threadIdx.x & 31).
static __device__ __forceinline__ void hiz_tail_warp(const HizJob& J) { hiz_tail<1, 3>(J); }

// Level 0 of tile `tile` of job J into v (4x4 per thread; 256 threads cover 64x64);
// outside the image the block reads 0 (those texels are never used).
__device__ __forceinline__ void hiz_tile_load(const HizJob& J, uint32_t tile, float (&v)[4][4]) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile_y = tile / J.tiles_x, tile_x = tile - tile_y * J.tiles_x;
    const uint32_t X0 = tile_x * kHizTile, Y0 = tile_y * kHizTile;
    const uint32_t W = J.lw[0], H = J.lh[0];
    const int tx4 = lane & 15, ty4 = warp * 2 + (lane >> 4);
    const uint32_t bx = X0 + 4 * tx4, by = Y0 + 4 * ty4;
    const bool aligned = ((J.depth_pitch & 3u) == 0u) && ((reinterpret_cast<uintptr_t>(J.depth) & 15u) == 0u);
    if (aligned && bx + 4 <= W && by + 4 <= H) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
            float4 q = __ldcs(reinterpret_cast<const float4*>(J.depth + (size_t)(by + r) * J.depth_pitch + bx));
            v[r][0] = q.x;
            v[r][1] = q.y;
            v[r][2] = q.z;
            v[r][3] = q.w;
        }
    } else {
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = 0; c < 4; ++c)
                v[r][c] = (bx + c < W && by + r < H) ? __ldcs(J.depth + (size_t)(by + r) * J.depth_pitch + bx + c) : 0.0f;
    }
}

// Level 0 of a loaded tile into the pyramid, when the job does not alias it.
__device__ __forceinline__ void hiz_tile_copy0(const HizJob& J, uint32_t tile, const float (&v)[4][4]) {
    if (!J.copy_mip0) return;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile_y = tile / J.tiles_x, tile_x = tile - tile_y * J.tiles_x;
    const uint32_t W = J.lw[0], H = J.lh[0];
    const uint32_t bx = tile_x * kHizTile + 4 * (lane & 15), by = tile_y * kHizTile + 4 * (warp * 2 + (lane >> 4));
    float* L0 = J.levels[0];
    const uint32_t p0 = J.lpitch[0];
    const bool al0 = ((p0 & 3u) == 0u) && ((reinterpret_cast<uintptr_t>(L0) & 15u) == 0u);
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        if (by + r >= H) break;
        float* row = L0 + (size_t)(by + r) * p0 + bx;
        if (al0 && bx + 4 <= W) {
            *reinterpret_cast<float4*>(row) = make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (bx + c < W) row[c] = v[r][c];
        }
    }
}

// Levels 1..3 of a loaded tile by all 256 threads (no barrier): level 3 goes to the
// pyramid and to s_m3 (8x9 shared) for levels 4..6.
__device__ __forceinline__ void hiz_tile_levels123(const HizJob& J, uint32_t tile, const float (&v)[4][4],
                                                   float (*s_m3)[9]) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint32_t tile_y = tile / J.tiles_x, tile_x = tile - tile_y * J.tiles_x;
    const uint32_t X0 = tile_x * kHizTile, Y0 = tile_y * kHizTile;
    const int tx4 = lane & 15, ty4 = warp * 2 + (lane >> 4);
    if (J.mip_count <= 1) return;
    // Level 1: 2x2 per thread.
    float m1[2][2];
    {
        const bool xc = J.lw[0] == 1u, yc = J.lh[0] == 1u;
#pragma unroll
        for (int j = 0; j < 2; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i)
                m1[j][i] = hiz_red4(v[2 * j][2 * i], v[2 * j][2 * i + 1], v[2 * j + 1][2 * i], v[2 * j + 1][2 * i + 1],
                                    xc, yc);
        const uint32_t x1 = (X0 >> 1) + 2 * tx4, y1 = (Y0 >> 1) + 2 * ty4;
        float* L1 = J.levels[1];
        const uint32_t p1 = J.lpitch[1];
#pragma unroll
        for (int j = 0; j < 2; ++j) {
            if (y1 + j >= J.lh[1]) break;
            float* row = L1 + (size_t)(y1 + j) * p1 + x1;
            if (x1 + 2 <= J.lw[1] && ((p1 & 1u) == 0u)) {
                *reinterpret_cast<float2*>(row) = make_float2(m1[j][0], m1[j][1]);
            } else {
                if (x1 < J.lw[1]) row[0] = m1[j][0];
                if (x1 + 1 < J.lw[1]) row[1] = m1[j][1];
            }
        }
    }
    if (J.mip_count <= 2) return;
    // Level 2: one texel per thread.
    const float m2 = hiz_red4(m1[0][0], m1[0][1], m1[1][0], m1[1][1], J.lw[1] == 1u, J.lh[1] == 1u);
    {
        const uint32_t x2 = (X0 >> 2) + tx4, y2 = (Y0 >> 2) + ty4;
        if (x2 < J.lw[2] && y2 < J.lh[2]) J.levels[2][(size_t)y2 * J.lpitch[2] + x2] = m2;
    }
    if (J.mip_count <= 3) return;
    // Level 3: 2x2 across lanes (x: lane^1, y: lane^16).
    float b = __shfl_xor_sync(0xffffffffu, m2, 1);
    float c = __shfl_xor_sync(0xffffffffu, m2, 16);
    float d = __shfl_xor_sync(0xffffffffu, m2, 17);
    float m3 = hiz_red4(m2, b, c, d, J.lw[2] == 1u, J.lh[2] == 1u);
    if ((lane & 17) == 0) {
        const int lx = tx4 >> 1, ly = warp;  // ty4 >> 1 == warp
        s_m3[ly][lx] = m3;
        const uint32_t x3 = (X0 >> 3) + lx, y3 = (Y0 >> 3) + ly;
        if (x3 < J.lw[3] && y3 < J.lh[3]) J.levels[3][(size_t)y3 * J.lpitch[3] + x3] = m3;
    }
}

// Levels 4..6 of a tile by one warp (lane = threadIdx.x & 31), from s_m3.
__device__ __forceinline__ void hiz_tile_levels456(const HizJob& J, uint32_t tile, const float (*s_m3)[9]) {
    const int lane = threadIdx.x & 31;
    const uint32_t tile_y = tile / J.tiles_x, tile_x = tile - tile_y * J.tiles_x;
    const uint32_t X0 = tile_x * kHizTile, Y0 = tile_y * kHizTile;
    if (J.mip_count <= 4) return;
    const int x4 = lane & 3, y4 = (lane >> 2) & 3;
    float m4 = hiz_red4(s_m3[2 * y4][2 * x4], s_m3[2 * y4][2 * x4 + 1], s_m3[2 * y4 + 1][2 * x4],
                        s_m3[2 * y4 + 1][2 * x4 + 1], J.lw[3] == 1u, J.lh[3] == 1u);
    if (lane < 16) {
        const uint32_t gx = (X0 >> 4) + x4, gy = (Y0 >> 4) + y4;
        if (gx < J.lw[4] && gy < J.lh[4]) J.levels[4][(size_t)gy * J.lpitch[4] + gx] = m4;
    }
    if (J.mip_count <= 5) return;
    float b = __shfl_xor_sync(0xffffffffu, m4, 1);
    float c = __shfl_xor_sync(0xffffffffu, m4, 4);
    float d = __shfl_xor_sync(0xffffffffu, m4, 5);
    float m5 = hiz_red4(m4, b, c, d, J.lw[4] == 1u, J.lh[4] == 1u);
    if (lane < 16 && (lane & 5) == 0) {
        const uint32_t gx = (X0 >> 5) + (x4 >> 1), gy = (Y0 >> 5) + (y4 >> 1);
        if (gx < J.lw[5] && gy < J.lh[5]) J.levels[5][(size_t)gy * J.lpitch[5] + gx] = m5;
    }
    if (J.mip_count <= 6) return;
    float b6 = __shfl_sync(0xffffffffu, m5, 2);
    float c6 = __shfl_sync(0xffffffffu, m5, 8);
    float d6 = __shfl_sync(0xffffffffu, m5, 10);
    float m6 = hiz_red4(m5, b6, c6, d6, J.lw[5] == 1u, J.lh[5] == 1u);
    if (lane == 0) {
        const uint32_t gx = X0 >> 6, gy = Y0 >> 6;
        if (gx < J.lw[6] && gy < J.lh[6]) J.levels[6][(size_t)gy * J.lpitch[6] + gx] = m6;
    }
}

// Warp 0, after its tile's level 6 is written: level 6 is written by warp 0 only, so
// warp 0 alone takes the job's ticket; the warp of the last tile of the job (over all
// CTAs) builds levels 7.. from level 6 and leaves the ticket at zero.
__device__ __forceinline__ void hiz_ticket_tail(const HizJob& J, uint32_t job, uint32_t* tickets) {
    const int lane = threadIdx.x & 31;
    __threadfence();
    __syncwarp();
    uint32_t last = 0u;
    if (lane == 0) {
        const uint32_t tiles = J.tiles_x * J.tiles_y;
        const uint32_t t = atomicAdd(&tickets[job], 1u);
        last = (t + 1 == tiles) ? 1u : 0u;
        if (last) tickets[job] = 0u;  // every other tile of this job has already taken its ticket
    }
    last = __shfl_sync(0xffffffffu, last, 0);
    if (last) {
        __threadfence();
        hiz_tail_warp(J);
    }
}

// Tile `tile` (flat index within job J, whose ticket is tickets[job]) by all 256
// threads of the CTA. s_m3 is an 8x9 shared scratch. Warps 1..7 return right
// after the level-3 barrier; warp 0 finishes levels 4..6 and, if this CTA is the
// last of the view, the tail. With tickets == nullptr the tile stops at level 6
// and the caller builds the tail after a grid-wide barrier.
__device__ __forceinline__ void hiz_tile(const HizJob& J, uint32_t job, uint32_t tile, uint32_t* tickets,
                                         float (*s_m3)[9]) {
    float v[4][4];
    hiz_tile_load(J, tile, v);
    hiz_tile_copy0(J, tile, v);
    if (J.mip_count <= 1) return;
    hiz_tile_levels123(J, tile, v, s_m3);
    if (J.mip_count <= 3) return;
    __syncthreads();
    if ((threadIdx.x >> 5) != 0) return;  // levels 4.. and the tail need only warp 0
    hiz_tile_levels456(J, tile, s_m3);
    if (J.mip_count <= 7 || tickets == nullptr) return;
    hiz_ticket_tail(J, job, tickets);
}

// ── Warp per 32x32 quadrant ─────────────────────────────────────────────────
// Warp q (0..3; q = 2 * row + column) of a tile reduces quadrant q alone: lane l holds
// the 8-row x 4-column block at quadrant column 4 (l % 8), row 8 (l / 8); registers give
// levels 1 and 2, shuffles levels 3..5, and the four quadrants' level-5 texels give
// level 6 (hiz_quad_level6, one thread, after a barrier). Each 2x2 step takes its texels
// in the order of the 4x4-per-thread form above (top-left, top-right, bottom-left,
// bottom-right) through hiz_red4, so both forms give identical pyramids.

// Level 0 of the lane's 8x4 block of quadrant q of tile `tile` from global memory;
// outside the image the block reads 0 (those texels are never used).
__device__ __forceinline__ void hiz_quad_load(const HizJob& J, uint32_t tile, int q, float (&v)[8][4]) {
    const int lane = threadIdx.x & 31;
    const uint32_t tile_y = tile / J.tiles_x, tile_x = tile - tile_y * J.tiles_x;
    const uint32_t bx = tile_x * kHizTile + 32u * (q & 1) + 4u * (lane & 7);
    const uint32_t by = tile_y * kHizTile + 32u * (q >> 1) + 8u * (lane >> 3);
    const uint32_t W = J.lw[0], H = J.lh[0];
    const bool aligned = ((J.depth_pitch & 3u) == 0u) && ((reinterpret_cast<uintptr_t>(J.depth) & 15u) == 0u);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        const float* row = J.depth + (size_t)(by + r) * J.depth_pitch + bx;
        if (aligned && bx + 4 <= W && by + r < H) {
            const float4 x = __ldcs(reinterpret_cast<const float4*>(row));
            v[r][0] = x.x;
            v[r][1] = x.y;
            v[r][2] = x.z;
            v[r][3] = x.w;
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c) v[r][c] = (bx + c < W && by + r < H) ? __ldcs(row + c) : 0.0f;
        }
    }
}

// Level 0 of the lane's 8x4 block of quadrant q of the tile at (X0, Y0) into the pyramid,
// when the job does not alias it.
__device__ __forceinline__ void hiz_quad_copy0(const HizJob& J, uint32_t X0, uint32_t Y0, int q,
                                               const float (&v)[8][4]) {
    if (!J.copy_mip0) return;
    const int lane = threadIdx.x & 31;
    const uint32_t bx = X0 + 32u * (q & 1) + 4u * (lane & 7), by = Y0 + 32u * (q >> 1) + 8u * (lane >> 3);
    const uint32_t W = J.lw[0], H = J.lh[0], p0 = J.lpitch[0];
    float* L0 = J.levels[0];
    const bool al0 = ((p0 & 3u) == 0u) && ((reinterpret_cast<uintptr_t>(L0) & 15u) == 0u);
#pragma unroll
    for (int r = 0; r < 8; ++r) {
        if (by + r >= H) break;
        float* row = L0 + (size_t)(by + r) * p0 + bx;
        if (al0 && bx + 4 <= W) {
            *reinterpret_cast<float4*>(row) = make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
        } else {
#pragma unroll
            for (int c = 0; c < 4; ++c)
                if (bx + c < W) row[c] = v[r][c];
        }
    }
}

// Stores texel (x, y) of level l when it lies inside the level.
__device__ __forceinline__ void hiz_put(const HizJob& J, int l, uint32_t x, uint32_t y, float m) {
    if (x < J.lw[l] && y < J.lh[l]) J.levels[l][(size_t)y * J.lpitch[l] + x] = m;
}

// Levels 1..5 of quadrant q of the tile at (X0, Y0) from the lane's 8x4 block v (lane =
// 8 * block row + block column); returns the quadrant's level-5 texel in lane 0.
__device__ __forceinline__ float hiz_quad_levels(const HizJob& J, uint32_t X0, uint32_t Y0, int q,
                                                 const float (&v)[8][4]) {
    const int lane = threadIdx.x & 31, lx = lane & 7, ly = lane >> 3;
    const uint32_t qx = (uint32_t)(q & 1), qy = (uint32_t)(q >> 1);
    // Level 1: 4 rows x 2 columns per lane.
    float m1[4][2];
    {
        const bool xc = J.lw[0] == 1u, yc = J.lh[0] == 1u;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int i = 0; i < 2; ++i)
                m1[j][i] = hiz_red4(v[2 * j][2 * i], v[2 * j][2 * i + 1], v[2 * j + 1][2 * i],
                                    v[2 * j + 1][2 * i + 1], xc, yc);
        const uint32_t x1 = (X0 >> 1) + 16u * qx + 2u * lx, y1 = (Y0 >> 1) + 16u * qy + 4u * ly;
        float* L1 = J.levels[1];
        const uint32_t p1 = J.lpitch[1];
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            if (y1 + j >= J.lh[1]) break;
            float* row = L1 + (size_t)(y1 + j) * p1 + x1;
            if (x1 + 2 <= J.lw[1] && ((p1 & 1u) == 0u)) {
                *reinterpret_cast<float2*>(row) = make_float2(m1[j][0], m1[j][1]);
            } else {
                if (x1 < J.lw[1]) row[0] = m1[j][0];
                if (x1 + 1 < J.lw[1]) row[1] = m1[j][1];
            }
        }
    }
    if (J.mip_count <= 2) return 0.0f;
    // Level 2: 2 rows x 1 column per lane.
    float m2[2];
#pragma unroll
    for (int j = 0; j < 2; ++j) {
        m2[j] = hiz_red4(m1[2 * j][0], m1[2 * j][1], m1[2 * j + 1][0], m1[2 * j + 1][1], J.lw[1] == 1u,
                         J.lh[1] == 1u);
        hiz_put(J, 2, (X0 >> 2) + 8u * qx + lx, (Y0 >> 2) + 8u * qy + 2u * ly + j, m2[j]);
    }
    if (J.mip_count <= 3) return 0.0f;
    // Level 3: the right neighbour is lane + 1 (lanes with an even block column).
    const float r0 = __shfl_xor_sync(0xffffffffu, m2[0], 1);
    const float r1 = __shfl_xor_sync(0xffffffffu, m2[1], 1);
    const float m3 = hiz_red4(m2[0], r0, m2[1], r1, J.lw[2] == 1u, J.lh[2] == 1u);
    if ((lx & 1) == 0) hiz_put(J, 3, (X0 >> 3) + 4u * qx + (lx >> 1), (Y0 >> 3) + 4u * qy + ly, m3);
    if (J.mip_count <= 4) return 0.0f;
    // Level 4: right = lane + 2, below = lane + 8 (lanes with block column % 4 == 0 and
    // an even block row).
    const float b4 = __shfl_xor_sync(0xffffffffu, m3, 2);
    const float c4 = __shfl_xor_sync(0xffffffffu, m3, 8);
    const float d4 = __shfl_xor_sync(0xffffffffu, m3, 10);
    const float m4 = hiz_red4(m3, b4, c4, d4, J.lw[3] == 1u, J.lh[3] == 1u);
    if ((lx & 3) == 0 && (ly & 1) == 0)
        hiz_put(J, 4, (X0 >> 4) + 2u * qx + (lx >> 2), (Y0 >> 4) + 2u * qy + (ly >> 1), m4);
    if (J.mip_count <= 5) return 0.0f;
    // Level 5: right = lane + 4, below = lane + 16 (lane 0).
    const float b5 = __shfl_xor_sync(0xffffffffu, m4, 4);
    const float c5 = __shfl_xor_sync(0xffffffffu, m4, 16);
    const float d5 = __shfl_xor_sync(0xffffffffu, m4, 20);
    const float m5 = hiz_red4(m4, b5, c5, d5, J.lw[4] == 1u, J.lh[4] == 1u);
    if (lane == 0) hiz_put(J, 5, (X0 >> 5) + qx, (Y0 >> 5) + qy, m5);
    return m5;
}

// Level 6 of tile t from its four quadrants' level-5 texels (one thread).
__device__ __forceinline__ void hiz_quad_level6(const HizJob& J, uint32_t t, const float* l5) {
    const uint32_t ty = t / J.tiles_x, tx = t - ty * J.tiles_x;
    hiz_put(J, 6, tx, ty, hiz_red4(l5[0], l5[1], l5[2], l5[3], J.lw[5] == 1u, J.lh[5] == 1u));
}

}  // namespace helio
