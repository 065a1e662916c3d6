// kpax_device.cuh — device building blocks of the expansion step.
//
// Rounding contract with the CPU oracle (oracle/kpax_oracle.c):
//  - control draws, step counts, region ids, cell ids, goal distance and scores are computed
//    with explicitly rounded intrinsics (__fadd_rn/__fmul_rn/__fdiv_rn) so no multiply-add is
//    fused; they are bit-identical to the oracle for identical inputs;
//  - the double-integrator step is written the same way, so DI segments are bit-identical;
//  - Dubins and quadrotor RK4 use a branch-free sine/cosine (sincos_fast, within a few ulp of
//    CUDA's sincosf), tan as sin times the reciprocal cosine and the PTX approximate square root
//    and reciprocal, and spell out every rounding and fused multiply-add (so a step gives the same
//    bits in every kernel it is inlined into); they match the oracle within the propagation
//    tolerance.
#pragma once
#include <stdint.h>

#include "kpax_params.h"

namespace kpax {

// ------------------------------------------------------------------ Philox4x32-10
// Salmon et al., SC'11.  ctr = {index, iter, sub-stream, stream}, key = seed.
struct U4 {
    uint32_t x, y, z, w;
};

__device__ __forceinline__ U4 philox(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for(int r = 0; r < 10; ++r) {
        uint32_t hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
        uint32_t hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
        uint32_t n0 = hi1 ^ c1 ^ k0, n2 = hi0 ^ c3 ^ k1;
        c0 = n0, c1 = lo1, c2 = n2, c3 = lo0;
        k0 += 0x9E3779B9u, k1 += 0xBB67AE85u;
    }
    return {c0, c1, c2, c3};
}

// ((x >> 8) + 1) * 2^-24: exact, in (0, 1].
__device__ __forceinline__ float u01(uint32_t x) { return __uint2float_rn((x >> 8) + 1u) * 5.9604644775390625e-8f; }

// The six uniforms of a child: controls c0..c3, duration, frontier draw.
__device__ __forceinline__ void child_draws(const KParams& p, uint32_t stream, uint32_t iter, uint32_t index, float u[6])
{
    U4 a = philox(index, iter, 0u, stream, p.seed_lo, p.seed_hi);
    U4 b = philox(index, iter, 1u, stream, p.seed_lo, p.seed_hi);
    u[0] = u01(a.x), u[1] = u01(a.y), u[2] = u01(a.z), u[3] = u01(a.w);
    u[4] = u01(b.x), u[5] = u01(b.y);
}

__device__ __forceinline__ float reactivate_draw(const KParams& p, uint32_t stream, uint32_t iter, uint32_t index)
{
    return u01(philox(index, iter, 2u, stream, p.seed_lo, p.seed_hi).x);
}

// Goal-progress pruning of an accepted child (prune_updateFrontier_kernel, PruneKPAX.cu:466-498):
// kept when the Philox stream-5 uniform is below clamp(explorationBias + goalBias *
// clamp((d_parent - d_child) / progressScale + 1/2, 0, 1), EPSILON, 1).
__device__ __forceinline__ bool prune_keep(const KParams& p, float d_parent, float d_child, uint32_t stream, uint32_t iter,
                                           uint32_t index)
{
    const float prog = fminf(fmaxf(__fadd_rn(__fdiv_rn(__fsub_rn(d_parent, d_child), p.prune_scale), 0.5f), 0.0f), 1.0f);
    const float prob = fminf(fmaxf(__fadd_rn(p.prune_expl_bias, __fmul_rn(p.prune_goal_bias, prog)), p.eps), 1.0f);
    return u01(philox(index, iter, 5u, stream, p.seed_lo, p.seed_hi).x) < prob;
}

// ------------------------------------------------------------------ sine / cosine
// Branch-free sin and cos of one argument for |x| <= kTrigFastMax: Cody-Waite reduction by pi/2
// with pi/2 split in three parts (1.5703125 + 4.837512969970703125e-4 + 7.54978995489188216e-8),
// then the single-precision minimax polynomials of the Cephes library (S. L. Moshier, sinf.c /
// cosf.c) on [-pi/4, pi/4] and the quadrant map.  Straight-line code, so several calls interleave;
// outside the range the caller falls back to CUDA's sincosf.  Error bound checked against
// sincosf in tests/test_gpu_kernels.py.
constexpr float kTrigFastMax = 8192.0f;

__device__ __forceinline__ void sincos_fast(float x, float* sn, float* cs)
{
    const float n = rintf(x * 0.636619772367581343f);  // 2 / pi
    float r = fmaf(n, -1.5703125f, x);
    r = fmaf(n, -4.837512969970703125e-4f, r);
    r = fmaf(n, -7.54978995489188216e-8f, r);
    const float z = r * r;
    const float ps = fmaf(fmaf(fmaf(-1.9515295891e-4f, z, 8.3321608736e-3f), z, -1.6666654611e-1f), z * r, r);
    const float pc = fmaf(fmaf(fmaf(2.443315711809948e-5f, z, -1.388731625493765e-3f), z, 4.166664568298827e-2f), z * z,
                          fmaf(-0.5f, z, 1.0f));
    const int q = (int)n & 3;
    const float a = (q & 1) ? pc : ps, b = (q & 1) ? ps : pc;
    *sn = (q & 2) ? -a : a;
    *cs = ((q + 1) & 2) ? -b : b;
}

__device__ __forceinline__ void sincos_checked(float x, float* sn, float* cs)
{
    sincos_fast(x, sn, cs);
    if(!(fabsf(x) <= kTrigFastMax)) sincosf(x, sn, cs);  // huge or non-finite arguments
}

// sin and cos of a0 + d from s0 = sin(a0), c0 = cos(a0) by the angle-sum identity, with the
// Taylor series of sin(d) to d^7 and cos(d) - 1 to d^8: for |d| <= kShiftMax the truncation error
// is below 2e-11, so the result is within a few ulp of sin/cos of the rounded sum a0 + d.  The RK4
// stages evaluate the attitude at a0 + (h/2) k and a0 + h k; this replaces three of every four
// full evaluations per angle and step.
constexpr float kShiftMax = 0.25f;
struct ShiftCoef {
    float sd, cm;  // sin(d) and cos(d) - 1
};

__device__ __forceinline__ ShiftCoef shift_coef(float d)
{
    const float d2 = d * d;
    return {fmaf(d * d2, fmaf(d2, fmaf(d2, -1.0f / 5040.0f, 1.0f / 120.0f), -1.0f / 6.0f), d),
            d2 * fmaf(d2, fmaf(d2, fmaf(d2, 1.0f / 40320.0f, -1.0f / 720.0f), 1.0f / 24.0f), -0.5f)};
}

__device__ __forceinline__ void sincos_apply(float s0, float c0, ShiftCoef k, float* sn, float* cs)
{
    *sn = fmaf(s0, k.cm, fmaf(c0, k.sd, s0));
    *cs = fmaf(c0, k.cm, fmaf(-s0, k.sd, c0));
}

__device__ __forceinline__ void sincos_shift(float s0, float c0, float d, float* sn, float* cs)
{
    sincos_apply(s0, c0, shift_coef(d), sn, cs);
}

// Square root and reciprocal by the PTX approximations sqrt.approx.f32 / rcp.approx.f32 (about one
// ulp, against the half ulp of the correctly rounded forms, which cost a Newton step and a
// special-case branch each): the quadrotor right-hand side takes two roots and one reciprocal
// per stage on its dependency chain.
__device__ __forceinline__ float sqrt_approx(float x)
{
    float y;
    asm("sqrt.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

__device__ __forceinline__ float rcp_approx(float x)
{
    float y;
    asm("rcp.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// float -> int with the reference's device semantics (saturating, NaN -> 0).
__device__ __forceinline__ int f2i(float x) { return __float2int_rz(x); }
__device__ __forceinline__ int clampi(int v, int lo, int hi) { return min(max(v, lo), hi); }

// ------------------------------------------------------------------ regions (Graph.cu:99-205)
// state s: the first 3 + cdim + vdim floats are read.  The attitude and velocity digits are
// visited with compile-time state indices (j < SD, predicated on the runtime dimensions) so the
// state stays in registers; the mixed-radix ids are the same integers as the reference's loops.
template <int SD>
__device__ __forceinline__ int region_r1(const KParams& p, const float* s)
{
    int w = 0, f = 1;
#pragma unroll
    for(int i = 2; i >= 0; --i) {
        int idx = f2i(__fdiv_rn(__fmul_rn((float)p.W1, __fsub_rn(s[i], p.wmin)), p.wspan));
        w += f * clampi(idx, 0, p.W1 - 1);
        f *= p.W1;
    }
    if(p.w_only) return w;
    int a = 0, v = 0;
    const int ce = 3 + p.cdim, ve = ce + p.vdim;
    if(p.C1 > 1) {  // digit i = j - 3, the last one least significant
#pragma unroll
        for(int j = 3; j < SD; ++j) {
            if(j < ce) {
                const float x = s[j];
                int idx = 0;
                for(int k = 0; k < p.C1 - 1; ++k) idx += (x >= p.cthr1[k]);
                a = a * p.C1 + idx;
            }
        }
    }
    if(p.V1 > 1) {
#pragma unroll
        for(int j = 3; j < SD; ++j) {
            if(j >= ce && j < ve) {
                int idx = f2i(__fdiv_rn(__fmul_rn((float)p.V1, __fsub_rn(s[j], p.vmin_r)), p.vspan));
                v = v * p.V1 + clampi(idx, 0, p.V1 - 1);
            }
        }
    }
    return w * p.r1_mulW + a * p.r1_mulA + v;
}

// getSubRegion (Graph.cu:155-205).  The R1 min corner is W_MIN + i*W_R1_SIZE (float),
// C_MIN + i*C_R1_SIZE (double, tabulated) and V_MIN + i*V_R1_SIZE (float), as Graph.cu:69-95.
// The R1 id's cell digits are decoded as they are consumed, least significant first.  In compat
// mode the id is decoded the way initializeRegions_kernel lays out its table (Graph.cu:58-96:
// workspace part fastest, C_R1^2 attitude cells, then velocity); otherwise in getRegion's order
// (workspace part slowest).
template <int SD>
__device__ __forceinline__ int region_r2(const KParams& p, const float* s, int r1)
{
    int wr, ar, vr;
    if(p.compat) {
        const int W3 = p.W1 * p.W1 * p.W1;
        wr = r1 % W3;
        ar = (r1 / W3) % (p.C1 * p.C1);
        vr = (r1 / (W3 * p.C1 * p.C1)) % p.V1;
    } else {
        wr = r1 / p.r1_mulW;
        const int rem = r1 - wr * p.r1_mulW;
        ar = rem / p.r1_mulA;
        vr = rem - ar * p.r1_mulA;
    }
    int w = 0, f = 1;
#pragma unroll
    for(int i = 2; i >= 0; --i) {
        const int dw = wr % p.W1;
        wr /= p.W1;
        const float m = __fadd_rn(p.wmin, __fmul_rn((float)dw, p.w1size));
        int idx = f2i(__fdiv_rn(__fmul_rn((float)p.W2, __fsub_rn(s[i], m)), p.w1size));
        w += f * clampi(idx, 0, p.W2 - 1);
        f *= p.W2;
    }
    int a = 0, v = 0;
    const int ce = 3 + p.cdim, ve = ce + p.vdim;
    if(p.C2 > 1) {
        f = 1;
#pragma unroll
        for(int j = SD - 1; j >= 3; --j) {
            if(j < ce) {
                const int da = ar % p.C1;
                ar /= p.C1;
                const float x = __fmul_rn((float)p.C2, __fsub_rn(s[j], p.cmin_tab[da]));
                int idx = 0;
                for(int k = 0; k < p.C2 - 1; ++k) idx += (x >= p.cthr2[k]);
                a += f * idx;
                f *= p.C2;
            }
        }
    }
    if(p.V2 > 1) {
        f = 1;
#pragma unroll
        for(int j = SD - 1; j >= 3; --j) {
            if(j >= ce && j < ve) {
                const int dv = vr % p.V1;
                vr /= p.V1;
                const float m = __fadd_rn(p.vmin_r, __fmul_rn((float)dv, p.v1size));
                int idx = f2i(__fdiv_rn(__fmul_rn((float)p.V2, __fsub_rn(s[j], m)), p.v1size));
                v += f * clampi(idx, 0, p.V2 - 1);
                f *= p.V2;
            }
        }
    }
    return r1 * p.P + (w * p.r2_mulW + a * p.r2_mulA + v);
}

// ------------------------------------------------------------------ spatial hash
// CSR grid over the workspace cube; obstacles as float4 pairs (min xyz, max xyz).
struct Grid {
    const float4* __restrict__ obs;
    const uint32_t* __restrict__ off;  // cells + 1
    const uint32_t* __restrict__ ent;
    float wmin, inv_cell;  // 1 / GRID_CELL_SIZE
    int dim;
};

// Cell of a coordinate.  Any non-decreasing map gives the brute-force verdict as long as the
// build and the query use the same one; a multiply by the reciprocal replaces the reference's
// division (spatialHash.cuh:236-246), which can move a point on a cell face by one cell.
__device__ __forceinline__ int grid_coord(const Grid& g, float x)
{
    return clampi(f2i(__fmul_rn(__fsub_rn(x, g.wmin), g.inv_cell)), 0, g.dim - 1);
}

// isMotionValidSpatialHash (spatialHash.cu:145-194) with isBroadPhaseValid (collisionCheck.cu:3-10):
// true when no obstacle overlaps the box strictly in all three dimensions.
// The box's cells are x0..x1, y0..y1, z0..z1.
__device__ __forceinline__ bool box_free_cells(const Grid& g, const float lo[3], const float hi[3], int x0, int y0, int z0,
                                               int x1, int y1, int z1)
{
    for(int gz = z0; gz <= z1; ++gz)
        for(int gy = y0; gy <= y1; ++gy)
            for(int gx = x0; gx <= x1; ++gx) {
                const int c = gx + g.dim * (gy + g.dim * gz);
                const uint32_t b = __ldg(g.off + c), e = __ldg(g.off + c + 1);
                for(uint32_t k = b; k < e; ++k) {
                    const uint32_t o = __ldg(g.ent + k);
                    const float4 a = __ldg(g.obs + 2 * o), m = __ldg(g.obs + 2 * o + 1);
                    if(hi[0] > a.x && m.x > lo[0] && hi[1] > a.y && m.y > lo[1] && hi[2] > a.z && m.z > lo[2]) return false;
                }
            }
    return true;
}

__device__ __forceinline__ bool box_free(const Grid& g, const float lo[3], const float hi[3])
{
    return box_free_cells(g, lo, hi, grid_coord(g, lo[0]), grid_coord(g, lo[1]), grid_coord(g, lo[2]), grid_coord(g, hi[0]),
                          grid_coord(g, hi[1]), grid_coord(g, hi[2]));
}

// The swept box of one step, p0 -> p1.  cells (optional): the cell coordinates of p0 on entry,
// replaced by p1's — a step's end is the next step's start, and since the cell map is
// non-decreasing the box's cell range is the range of its two corners' cells, so each step maps
// one point instead of two.
__device__ __forceinline__ bool step_free(const Grid& g, const float p0[3], const float p1[3], int* cells = nullptr)
{
    float lo[3], hi[3];
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        const bool sw = p0[d] > p1[d];
        lo[d] = sw ? p1[d] : p0[d];
        hi[d] = sw ? p0[d] : p1[d];
    }
    if(!cells) return box_free(g, lo, hi);
    const int c1[3] = {grid_coord(g, p1[0]), grid_coord(g, p1[1]), grid_coord(g, p1[2])};
    const bool ok = box_free_cells(g, lo, hi, min(cells[0], c1[0]), min(cells[1], c1[1]), min(cells[2], c1[2]),
                                   max(cells[0], c1[0]), max(cells[1], c1[1]), max(cells[2], c1[2]));
    cells[0] = c1[0], cells[1] = c1[1], cells[2] = c1[2];
    return ok;
}

// x * 0 is +-0 for a finite x and NaN for an infinite or NaN one, so the sum of those products is
// 0 exactly when every value is finite (two chains for a shorter dependency).
__device__ __forceinline__ bool finite_all(const float* s, int n)
{
    float a = 0.0f, b = 0.0f;
#pragma unroll
    for(int i = 0; i + 1 < n; i += 2) a = __fmaf_rn(s[i], 0.0f, a), b = __fmaf_rn(s[i + 1], 0.0f, b);
    if(n & 1) a = __fmaf_rn(s[n - 1], 0.0f, a);
    return __fadd_rn(a, b) == 0.0f;
}

// ------------------------------------------------------------------ controls
// statePropagatorSpatialHash.cu:74-77 / 141-144 / 236-241: c = MIN + u * (MAX - MIN);
// steps = 1 + (int)(u * N) (N + 1 when u == 1, as in the reference).
__device__ __forceinline__ int draw_controls(const KParams& p, const float u[6], float c[4])
{
#pragma unroll
    for(int i = 0; i < 4; ++i) c[i] = __fadd_rn(p.clo[i], __fmul_rn(u[i], p.crng[i]));
    return p.fixed_steps ? p.nsteps : 1 + f2i(__fmul_rn(u[4], (float)p.nsteps));
}

// ------------------------------------------------------------------ models
// One integration step per model with the reference's per-step checks, in the reference's order
// (bounds, then the swept box's collision query); the output row holds the state after the
// failing step, as the reference's break does.

// The configuration values a step reads, copied to registers once per segment (the planner keeps
// its KParams in shared memory).
struct StepParams {
    float h, hh, h6, vmin, vmax, ws_lo, ws_hi, pitch_lo, pitch_hi;
};

__device__ __forceinline__ StepParams step_params(const KParams& p)
{
    return {p.h, p.hh, p.h6, p.vmin, p.vmax, p.ws_lo, p.ws_hi, p.pitch_lo, p.pitch_hi};
}

// Double integrator, statePropagatorSpatialHash.cu:72-134 (x += h(5v + 2ah)/6, not textbook RK4).  The terms
// that depend on the segment's acceleration only (a*h/2, a*h and the velocity increment
// (a + 2a + 2a + a)*h/6) are computed once per segment, with the same rounded operations.
struct DIConsts {
    float ah2[3], ah[3], dv[3];
};

__device__ __forceinline__ DIConsts di_consts(const KParams& p, const float* c)
{
    DIConsts k;
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        const float a = c[d];
        k.ah[d] = __fmul_rn(a, p.h);
        k.ah2[d] = __fdiv_rn(k.ah[d], 2.0f);
        const float asum = __fadd_rn(__fadd_rn(__fadd_rn(a, __fmul_rn(2.0f, a)), __fmul_rn(2.0f, a)), a);
        k.dv[d] = __fdiv_rn(__fmul_rn(asum, p.h), 6.0f);
    }
    return k;
}

// One step from s in place; false when the step fails a check (velocity box, workspace, finite,
// collision).
__device__ __forceinline__ bool step_di(const StepParams& p, const Grid& g, float* s, const DIConsts& k, int* cells = nullptr)
{
    const float h = p.h;
    const float p0[3] = {s[0], s[1], s[2]};
#pragma unroll
    for(int d = 0; d < 3; ++d) {
        const float v = s[3 + d];
        // (v + (v + 2*(v + a*h/2) + (v + a*h))) * h / 6
        const float t1 = __fadd_rn(v, k.ah2[d]);
        const float t2 = __fadd_rn(v, k.ah[d]);
        const float sum = __fadd_rn(v, __fadd_rn(__fadd_rn(v, __fmul_rn(2.0f, t1)), t2));
        s[d] = __fadd_rn(s[d], __fdiv_rn(__fmul_rn(sum, h), 6.0f));
        s[3 + d] = __fadd_rn(v, k.dv[d]);  // v + (a + 2a + 2a + a) * h / 6
    }
    if(s[3] < p.vmin || s[3] > p.vmax || s[4] < p.vmin || s[4] > p.vmax || s[5] < p.vmin || s[5] > p.vmax) return false;
    if(s[0] < p.ws_lo || s[0] > p.ws_hi || s[1] < p.ws_lo || s[1] > p.ws_hi || s[2] < p.ws_lo || s[2] > p.ws_hi) return false;
    return finite_all(s, 6) && step_free(g, p0, s, cells);
}

// Dubins airplane, statePropagatorSpatialHash.cu:139-229; c = (a, yawRate, pitchRate).  One step
// from s in place; false when the step fails a check (speed, pitch range, workspace, finite, collision).
// The stage angle increments of a Dubins segment are its fixed rates times h/2 and h, so their
// sine / cosine series are evaluated once per segment.
struct DubinsShifts {
    bool shift;  // all four increments within kShiftMax
    ShiftCoef p1, y1, p2, y2;
};

__device__ __forceinline__ DubinsShifts dubins_shifts(const KParams& p, const float* c)
{
    const float h = p.h, hh = p.hh, yr = c[1], pr = c[2];
    return {fmaxf(fabsf(__fmul_rn(h, pr)), fabsf(__fmul_rn(h, yr))) <= kShiftMax, shift_coef(__fmul_rn(hh, pr)),
            shift_coef(__fmul_rn(hh, yr)), shift_coef(__fmul_rn(h, pr)), shift_coef(__fmul_rn(h, yr))};
}

__device__ __forceinline__ bool step_dubins(const StepParams& p, const Grid& g, float* s, const float* c, const DubinsShifts& k,
                                            int* cells = nullptr)
{
    const float h = p.h, hh = p.hh, h6 = p.h6;
    const float a = c[0], yr = c[1], pr = c[2];
    const float p0[3] = {s[0], s[1], s[2]};
    const float yaw = s[3], pitch = s[4], v = s[5];
    float sp0, cp0, sy0, cy0, sp1, cp1, sy1, cy1, sp2, cp2, sy2, cy2;
    sincos_checked(pitch, &sp0, &cp0);
    sincos_checked(yaw, &sy0, &cy0);
    if(k.shift) {
        sincos_apply(sp0, cp0, k.p1, &sp1, &cp1);
        sincos_apply(sy0, cy0, k.y1, &sy1, &cy1);
        sincos_apply(sp0, cp0, k.p2, &sp2, &cp2);
        sincos_apply(sy0, cy0, k.y2, &sy2, &cy2);
    } else {
        sincos_checked(__fmaf_rn(hh, pr, pitch), &sp1, &cp1);
        sincos_checked(__fmaf_rn(hh, yr, yaw), &sy1, &cy1);
        sincos_checked(__fmaf_rn(h, pr, pitch), &sp2, &cp2);
        sincos_checked(__fmaf_rn(h, yr, yaw), &sy2, &cy2);
    }
    // every rounding written out (as the quadrotor's): the same bits wherever the step is inlined
    const float vm = __fmaf_rn(hh, a, v), ve = __fmaf_rn(h, a, v);
    const float vmc = __fmul_rn(vm, cp1), vc0 = __fmul_rn(v, cp0), vc2 = __fmul_rn(ve, cp2);
    const float mx = __fmul_rn(vmc, cy1), my = __fmul_rn(vmc, sy1), mz = __fmul_rn(vm, sp1);
    // (k1 + 2 (k2 + k3)) + k4 with k2 = k3 (the reference's stage sum; 2 x is exact)
    s[0] = __fmaf_rn(h6, __fmaf_rn(vc2, cy2, __fmaf_rn(2.0f, __fadd_rn(mx, mx), __fmul_rn(vc0, cy0))), s[0]);
    s[1] = __fmaf_rn(h6, __fmaf_rn(vc2, sy2, __fmaf_rn(2.0f, __fadd_rn(my, my), __fmul_rn(vc0, sy0))), s[1]);
    s[2] = __fmaf_rn(h6, __fmaf_rn(ve, sp2, __fmaf_rn(2.0f, __fadd_rn(mz, mz), __fmul_rn(v, sp0))), s[2]);
    s[3] = __fmaf_rn(h, yr, yaw);
    s[4] = __fmaf_rn(h, pr, pitch);
    s[5] = __fmaf_rn(h6, __fadd_rn(__fmaf_rn(2.0f, __fadd_rn(a, a), a), a), v);
    if(s[5] < p.vmin || s[5] > p.vmax || s[4] < p.pitch_lo || s[4] > p.pitch_hi) return false;
    if(s[0] < p.ws_lo || s[0] > p.ws_hi || s[1] < p.ws_lo || s[1] > p.ws_hi || s[2] < p.ws_lo || s[2] > p.ws_hi) return false;
    return finite_all(s, 6) && step_free(g, p0, s, cells);
}

// Quadrotor right-hand side, statePropagator.cu:325-370, in its two halves: the kinematics
// (position and Euler-angle rates, xd[0..5]) read the attitude's sines and cosines and the body
// velocities and rates; the dynamics (velocity and rate derivatives, xd[6..11]) read sin/cos of
// roll and pitch, the velocities, rates and controls.  Model constants NU 10e-3, MU 2e-6, IX 1,
// IY 1, IZ 2, GRAVITY -9.81, MASS 1 (config.h:300-308).  Every operation is written out (explicit
// roundings and fused multiply-adds), so the result does not depend on how the compiler contracts
// the expressions where the step is inlined.
struct QuadTrig {
    float sf, cf, st, ct, sp, cp;  // sin / cos of roll, pitch, yaw
};
struct QuadRates {
    float u, v, w, p, q, r;  // body velocities and rates
};

__device__ __forceinline__ void quad_kin(float* xd, const QuadTrig& t, const QuadRates& b)
{
    const float sec = rcp_approx(t.ct);  // tan(theta) = sin * sec, 1/cos(theta) = sec
    const float sfst = __fmul_rn(t.sf, t.st), cfst = __fmul_rn(t.cf, t.st);
    const float r01 = __fmaf_rn(sfst, t.cp, -__fmul_rn(t.cf, t.sp)), r02 = __fmaf_rn(cfst, t.cp, __fmul_rn(t.sf, t.sp));
    const float r11 = __fmaf_rn(sfst, t.sp, __fmul_rn(t.cf, t.cp)), r12 = __fmaf_rn(cfst, t.sp, -__fmul_rn(t.sf, t.cp));
    xd[0] = __fmaf_rn(r02, b.w, __fmaf_rn(r01, b.v, __fmul_rn(__fmul_rn(t.ct, t.cp), b.u)));
    xd[1] = __fmaf_rn(r12, b.w, __fmaf_rn(r11, b.v, __fmul_rn(__fmul_rn(t.ct, t.sp), b.u)));
    xd[2] = __fmaf_rn(__fmul_rn(t.cf, t.ct), b.w, __fmaf_rn(__fmul_rn(t.sf, t.ct), b.v, -__fmul_rn(t.st, b.u)));
    const float qr = __fmaf_rn(b.q, t.sf, __fmul_rn(b.r, t.cf));
    xd[3] = __fmaf_rn(qr, __fmul_rn(t.st, sec), b.p);
    xd[4] = __fmaf_rn(b.q, t.cf, -__fmul_rn(b.r, t.sf));
    xd[5] = __fmul_rn(qr, sec);
}

__device__ __forceinline__ void quad_dyn(float* xd, float sf, float cf, float st, float ct, const QuadRates& b, const float* c)
{
    const float NU = 10e-3f, MU = 2e-6f, G = -9.81f;
    const float XYZ = __fmul_rn(-NU, sqrt_approx(__fmaf_rn(b.w, b.w, __fmaf_rn(b.v, b.v, __fmul_rn(b.u, b.u)))));
    const float gct = __fmul_rn(G, ct);
    xd[0] = __fmaf_rn(XYZ, b.u, __fmaf_rn(-G, st, __fmaf_rn(b.r, b.v, -__fmul_rn(b.q, b.w))));
    xd[1] = __fmaf_rn(XYZ, b.v, __fmaf_rn(gct, sf, __fmaf_rn(b.p, b.w, -__fmul_rn(b.r, b.u))));
    xd[2] = __fadd_rn(__fmaf_rn(XYZ, b.w, __fmaf_rn(gct, cf, __fmaf_rn(b.q, b.u, -__fmul_rn(b.p, b.v)))), c[0]);
    const float LMN = __fmul_rn(-MU, sqrt_approx(__fmaf_rn(b.r, b.r, __fmaf_rn(b.q, b.q, __fmul_rn(b.p, b.p)))));
    xd[3] = __fadd_rn(__fmaf_rn(LMN, b.p, -__fmul_rn(b.q, b.r)), c[1]);  // (IY - IZ)/IX = -1, 1/IX = 1
    xd[4] = __fadd_rn(__fmaf_rn(LMN, b.q, __fmul_rn(b.p, b.r)), c[2]);   // (IZ - IX)/IY = 1,  1/IY = 1
    // (IX - IY)/IZ = 0 (the product still carries a non-finite rate), 1/IZ = 0.5
    xd[5] = __fmaf_rn(0.5f, c[3], __fmaf_rn(0.5f, __fmul_rn(LMN, b.r), __fmul_rn(0.0f, __fmul_rn(b.p, b.q))));
}

// The first RK4 stage is evaluated at x0 + 1 * 0: the state is x0 + 0 (which only turns -0 into
// +0) and the angle-sum shift by 0 reduces to sin + 0 and cos.  trig0: (sin, cos) of the three
// Euler angles of x0.
__device__ __forceinline__ QuadTrig quad_first_trig(const float* trig0)
{
    return {__fadd_rn(trig0[0], 0.0f), trig0[1], __fadd_rn(trig0[2], 0.0f), trig0[3], __fadd_rn(trig0[4], 0.0f), trig0[5]};
}

__device__ __forceinline__ QuadRates quad_first_rates(const float* v0)
{
    return {__fadd_rn(v0[0], 0.0f), __fadd_rn(v0[1], 0.0f), __fadd_rn(v0[2], 0.0f),
            __fadd_rn(v0[3], 0.0f), __fadd_rn(v0[4], 0.0f), __fadd_rn(v0[5], 0.0f)};
}

// The attitude at a0 + delta * ka (later stages): sin and cos by the angle-sum shift of trig0;
// large attitude increments or non-finite values are evaluated at the rounded angles.
__device__ __forceinline__ QuadTrig quad_stage_trig(const float* a0, const float* trig0, const float* ka, float delta)
{
    QuadTrig t;
    const float d0 = __fmul_rn(delta, ka[0]), d1 = __fmul_rn(delta, ka[1]), d2 = __fmul_rn(delta, ka[2]);
    if(fmaxf(fabsf(d0), fmaxf(fabsf(d1), fabsf(d2))) <= kShiftMax) {
        sincos_shift(trig0[0], trig0[1], d0, &t.sf, &t.cf);
        sincos_shift(trig0[2], trig0[3], d1, &t.st, &t.ct);
        sincos_shift(trig0[4], trig0[5], d2, &t.sp, &t.cp);
    } else {
        sincos_checked(__fadd_rn(a0[0], d0), &t.sf, &t.cf);
        sincos_checked(__fadd_rn(a0[1], d1), &t.st, &t.ct);
        sincos_checked(__fadd_rn(a0[2], d2), &t.sp, &t.cp);
    }
    return t;
}

__device__ __forceinline__ QuadRates quad_stage_rates(const float* v0, const float* kv, float delta)
{
    return {__fmaf_rn(delta, kv[0], v0[0]), __fmaf_rn(delta, kv[1], v0[1]), __fmaf_rn(delta, kv[2], v0[2]),
            __fmaf_rn(delta, kv[3], v0[3]), __fmaf_rn(delta, kv[4], v0[4]), __fmaf_rn(delta, kv[5], v0[5])};
}

__device__ __forceinline__ void quad_trig0(const float* a0, float* trig0)
{
    sincos_checked(a0[0], &trig0[0], &trig0[1]);
    sincos_checked(a0[1], &trig0[2], &trig0[3]);
    sincos_checked(a0[2], &trig0[4], &trig0[5]);
}

// The per-step checks of each half, in the reference's order (velocity box; workspace; then the
// finite check and the swept box's collision query).
// A box check of three values by their minimum and maximum: fminf / fmaxf pass over a NaN that the
// six comparisons would let through as well, and the finite check rejects it either way, so the
// verdict is the comparisons'.
__device__ __forceinline__ bool in_box3(const float* v, float lo, float hi)
{
    return !(fminf(fminf(v[0], v[1]), v[2]) < lo || fmaxf(fmaxf(v[0], v[1]), v[2]) > hi);
}

__device__ __forceinline__ bool quad_dyn_ok(const StepParams& p, const float* v)
{
    return in_box3(v, p.vmin, p.vmax) && finite_all(v, 6);
}

__device__ __forceinline__ bool quad_kin_ok(const StepParams& p, const Grid& g, const float* p0, const float* x,
                                            int* cells = nullptr)
{
    if(!in_box3(x, p.ws_lo, p.ws_hi)) return false;
    return finite_all(x, 6) && step_free(g, p0, x, cells);
}

// Quadrotor RK4, statePropagatorSpatialHash.cu:234-308: four stages, the stage sum in the
// reference's order ((k1 + 2k2) + 2k3) + k4.  One step from s in place; false when the step fails
// a check (velocity box, workspace, finite, collision).
__device__ __forceinline__ bool step_quad(const StepParams& p, const Grid& g, float* s, const float* c, int* cells = nullptr)
{
    const float h = p.h, hh = p.hh, h6 = p.h6;
    const float p0[3] = {s[0], s[1], s[2]};
    float k[12], acc[12], trig0[6];
    quad_trig0(s + 3, trig0);
    {
        const QuadTrig t = quad_first_trig(trig0);
        const QuadRates b = quad_first_rates(s + 6);
        quad_kin(k, t, b);
        quad_dyn(k + 6, t.sf, t.cf, t.st, t.ct, b, c);
    }
#pragma unroll
    for(int j = 0; j < 12; ++j) acc[j] = k[j];
#pragma unroll 1
    for(int stage = 1; stage < 4; ++stage) {
        const float delta = stage == 3 ? h : hh, w = stage == 3 ? 1.0f : 2.0f;
        const QuadTrig t = quad_stage_trig(s + 3, trig0, k + 3, delta);
        const QuadRates b = quad_stage_rates(s + 6, k + 6, delta);
        quad_kin(k, t, b);
        quad_dyn(k + 6, t.sf, t.cf, t.st, t.ct, b, c);
#pragma unroll
        for(int j = 0; j < 12; ++j) acc[j] = __fmaf_rn(w, k[j], acc[j]);
    }
#pragma unroll
    for(int j = 0; j < 12; ++j) s[j] = __fmaf_rn(h6, acc[j], s[j]);
    return quad_dyn_ok(p, s + 6) && quad_kin_ok(p, g, p0, s, cells);
}

// Per-segment constants of a model's step (the double integrator's acceleration terms, the Dubins
// stage shifts; nothing for the quadrotor).
struct NoSegmentConsts {};
template <int M>
__device__ __forceinline__ auto segment_consts(const KParams& p, const float* c)
{
    if constexpr(M == KPAX_MODEL_DUBINS_AIRPLANE) return dubins_shifts(p, c);
    else if constexpr(M == KPAX_MODEL_DOUBLE_INTEGRATOR) return di_consts(p, c);
    else return NoSegmentConsts{};
}

template <int M, class K>
__device__ __forceinline__ bool model_step(const StepParams& p, const Grid& g, float* s, const float* c, const K& k,
                                           int* cells = nullptr)
{
    if constexpr(M == KPAX_MODEL_DOUBLE_INTEGRATOR) return step_di(p, g, s, k, cells);
    else if constexpr(M == KPAX_MODEL_DUBINS_AIRPLANE) return step_dubins(p, g, s, c, k, cells);
    else return step_quad(p, g, s, c, cells);
}

// Propagates `steps` steps from s (in place), checking every step like the reference, and
// returns validity; `done` receives the number of steps executed (the failing one included).
template <int M>
__device__ __forceinline__ bool propagate(const KParams& p, const Grid& g, float* s, const float* c, int steps, int& done)
{
    const auto k = segment_consts<M>(p, c);
    const StepParams sp = step_params(p);
    const Grid gl = g;  // register copy of the grid's pointers and cell map
    int cells[3] = {grid_coord(gl, s[0]), grid_coord(gl, s[1]), grid_coord(gl, s[2])};  // of the current position
    for(int i = 0; i < steps; ++i) {
        if(!model_step<M>(sp, gl, s, c, k, cells)) {
            done = i + 1;
            return false;
        }
    }
    done = steps;
    return true;
}

template <int M>
struct ModelDims;
template <>
struct ModelDims<KPAX_MODEL_DOUBLE_INTEGRATOR> {
    static constexpr int SD = 6, CD = 3;
};
template <>
struct ModelDims<KPAX_MODEL_DUBINS_AIRPLANE> {
    static constexpr int SD = 6, CD = 3;
};
template <>
struct ModelDims<KPAX_MODEL_QUADROTOR> {
    static constexpr int SD = 12, CD = 4;
};

// Controls as stored in the row: Dubins stores (yawRate, pitchRate, a) (statePropagatorSpatialHash.cu:223-225).
template <int M>
__device__ __forceinline__ void row_controls(const float* c, float* out)
{
    if constexpr(M == KPAX_MODEL_DUBINS_AIRPLANE) {
        out[0] = c[1], out[1] = c[2], out[2] = c[0], out[3] = 0.0f;
    } else {
#pragma unroll
        for(int i = 0; i < 4; ++i) out[i] = c[i];
    }
}

}  // namespace kpax
