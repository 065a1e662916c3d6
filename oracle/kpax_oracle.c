/*
 * kpax_oracle.c — CPU restatement of the Kino-PAX tree-expansion iteration.
 * TEST INFRASTRUCTURE (see kpax_oracle.h): the checker for the CUDA path and the CPU baseline,
 * never called by the library.  Built with -ffp-contract=off so every float operation rounds
 * exactly where the reference's source rounds (no fused multiply-add).
 *
 * Reference citations are path:line inside the Kino-PAX-Fork tree.
 */
#define _GNU_SOURCE
#include "kpax_oracle.h"

#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define KO_PENDING 255u

/* ---------------------------------------------------------------- helpers ------------- */

/* float -> int as the reference's device code converts (cvt.rzi.s32: saturate, NaN -> 0). */
static int f2i(float x)
{
    if(x != x) return 0;
    if(x >= 2147483648.0f) return INT_MAX;
    if(x <= -2147483648.0f) return INT_MIN;
    return (int)x;
}

static int d2i(double x)
{
    if(x != x) return 0;
    if(x >= 2147483648.0) return INT_MAX;
    if(x <= -2147483648.0) return INT_MIN;
    return (int)x;
}

static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

static int ipow(int b, int e)
{
    int r = 1;
    while(e-- > 0) r *= b;
    return r;
}

static float minf_(float a, float b) { return (b < a || a != a) ? b : a; }

/* ---------------------------------------------------------------- Philox4x32-10 -------- */
/* Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy as 1, 2, 3", SC'11:
 * 10 rounds of two 32x32->64 multiplies with Weyl-sequence key schedule. */
void ko_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t x0 = ctr[0], x1 = ctr[1], x2 = ctr[2], x3 = ctr[3], k0 = key[0], k1 = key[1];
    for(int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * x0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * x2;
        uint32_t y0 = (uint32_t)(p1 >> 32) ^ x1 ^ k0;
        uint32_t y1 = (uint32_t)p1;
        uint32_t y2 = (uint32_t)(p0 >> 32) ^ x3 ^ k1;
        uint32_t y3 = (uint32_t)p0;
        x0 = y0, x1 = y1, x2 = y2, x3 = y3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = x0, out[1] = x1, out[2] = x2, out[3] = x3;
}

float ko_u01(uint32_t x) { return (float)((x >> 8) + 1u) * 5.9604644775390625e-8f; }

void ko_child_draws(uint64_t seed, uint32_t stream, uint32_t iter, uint32_t index, float u[6])
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t c0[4] = {index, iter, 0u, stream}, c1[4] = {index, iter, 1u, stream}, o[4];
    ko_philox4x32_10(c0, key, o);
    for(int i = 0; i < 4; ++i) u[i] = ko_u01(o[i]);
    ko_philox4x32_10(c1, key, o);
    u[4] = ko_u01(o[0]);
    u[5] = ko_u01(o[1]);
}

float ko_reactivate_draw(uint64_t seed, uint32_t stream, uint32_t iter, uint32_t index)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t c[4] = {index, iter, 2u, stream}, o[4];
    ko_philox4x32_10(c, key, o);
    return ko_u01(o[0]);
}

/* Goal-progress pruning draw (PruneKPAX.cu:488-489): Philox sub-stream 5. */
float ko_prune_draw(uint64_t seed, uint32_t stream, uint32_t iter, uint32_t index)
{
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    uint32_t c[4] = {index, iter, 5u, stream}, o[4];
    ko_philox4x32_10(c, key, o);
    return ko_u01(o[0]);
}

/* ---------------------------------------------------------------- sizes --------------- */

int ko_sizes(const kpax_config* cfg, uint32_t* num_r1, uint32_t* r2_per_r1, uint32_t* sample_dim)
{
    uint32_t n1 = (uint32_t)(ipow(cfg->w_r1_length, 3) * ipow(cfg->c_r1_length, cfg->c_dim) *
                             ipow(cfg->v_r1_length, cfg->v_dim));
    uint32_t p = (uint32_t)(ipow(cfg->w_r2_length, 3) * ipow(cfg->c_r2_length, cfg->c_dim) *
                            ipow(cfg->v_r2_length, cfg->v_dim));
    if(num_r1) *num_r1 = n1;
    if(r2_per_r1) *r2_per_r1 = p;
    if(sample_dim) *sample_dim = (uint32_t)(cfg->state_dim + cfg->control_dim + 1);
    return 0;
}

/* ---------------------------------------------------------------- collision ----------- */
/* Uniform grid over the workspace cube (spatialHash.cuh:9-13, 42-60), stored as CSR with
 * every (cell, obstacle) pair kept and ascending obstacle order inside a cell. */
struct ko_env {
    float* obs;
    uint32_t n;
    float wmin, cell;
    int dim;
    uint32_t* off;
    uint32_t* ent;
    uint32_t nent;
};

static int grid_coord(const ko_env* e, float x)
{
    return clampi(f2i((x - e->wmin) / e->cell), 0, e->dim - 1);
}

ko_env* ko_env_create(const kpax_config* cfg, const float* obs, uint32_t n)
{
    ko_env* e = (ko_env*)calloc(1, sizeof(ko_env));
    e->n = n;
    e->obs = (float*)malloc(sizeof(float) * 6 * (n ? n : 1));
    if(n) memcpy(e->obs, obs, sizeof(float) * 6 * n);
    e->wmin = cfg->w_min;
    e->cell = cfg->hash_cell_size;
    e->dim = (int)((cfg->w_max - cfg->w_min) / cfg->hash_cell_size) + 1;
    uint32_t cells = (uint32_t)(e->dim * e->dim * e->dim);
    e->off = (uint32_t*)calloc(cells + 1, sizeof(uint32_t));
    for(int pass = 0; pass < 2; ++pass) {
        uint32_t* cur = NULL;
        if(pass == 1) {
            uint32_t s = 0;
            for(uint32_t c = 0; c < cells; ++c) {
                uint32_t k = e->off[c];
                e->off[c] = s;
                s += k;
            }
            e->off[cells] = s;
            e->nent = s;
            e->ent = (uint32_t*)malloc(sizeof(uint32_t) * (s ? s : 1));
            cur = (uint32_t*)malloc(sizeof(uint32_t) * cells);
            memcpy(cur, e->off, sizeof(uint32_t) * cells);
        }
        for(uint32_t o = 0; o < n; ++o) {
            const float* b = e->obs + 6 * o;
            int x0 = grid_coord(e, b[0]), y0 = grid_coord(e, b[1]), z0 = grid_coord(e, b[2]);
            int x1 = grid_coord(e, b[3]), y1 = grid_coord(e, b[4]), z1 = grid_coord(e, b[5]);
            for(int gz = z0; gz <= z1; ++gz)
                for(int gy = y0; gy <= y1; ++gy)
                    for(int gx = x0; gx <= x1; ++gx) {
                        uint32_t c = (uint32_t)(gx + gy * e->dim + gz * e->dim * e->dim);
                        if(pass == 0) e->off[c]++;
                        else e->ent[cur[c]++] = o;
                    }
        }
        free(cur);
    }
    return e;
}

void ko_env_destroy(ko_env* e)
{
    if(!e) return;
    free(e->obs);
    free(e->off);
    free(e->ent);
    free(e);
}

void ko_env_grid(const ko_env* e, uint32_t* n_cells, uint32_t* n_entries, uint32_t* offsets, uint32_t* entries)
{
    uint32_t cells = (uint32_t)(e->dim * e->dim * e->dim);
    if(n_cells) *n_cells = cells;
    if(n_entries) *n_entries = e->nent;
    if(offsets) memcpy(offsets, e->off, sizeof(uint32_t) * (cells + 1));
    if(entries) memcpy(entries, e->ent, sizeof(uint32_t) * e->nent);
}

/* isBroadPhaseValid (collisionCheck.cu:3-10): free unless the boxes overlap strictly in all dims. */
static int broad_free(const float* bmin, const float* bmax, const float* o)
{
    for(int d = 0; d < 3; ++d)
        if(bmax[d] <= o[d] || o[3 + d] <= bmin[d]) return 1;
    return 0;
}

int ko_collide_brute(const float* obs, uint32_t n, const float bmin[3], const float bmax[3])
{
    for(uint32_t o = 0; o < n; ++o)
        if(!broad_free(bmin, bmax, obs + 6 * o)) return 0;
    return 1;
}

/* isMotionValidSpatialHash (spatialHash.cu:145-194) over the CSR grid. */
int ko_collide_hash(const ko_env* e, const float bmin[3], const float bmax[3])
{
    int x0 = grid_coord(e, bmin[0]), y0 = grid_coord(e, bmin[1]), z0 = grid_coord(e, bmin[2]);
    int x1 = grid_coord(e, bmax[0]), y1 = grid_coord(e, bmax[1]), z1 = grid_coord(e, bmax[2]);
    for(int gz = z0; gz <= z1; ++gz)
        for(int gy = y0; gy <= y1; ++gy)
            for(int gx = x0; gx <= x1; ++gx) {
                uint32_t c = (uint32_t)(gx + gy * e->dim + gz * e->dim * e->dim);
                for(uint32_t k = e->off[c]; k < e->off[c + 1]; ++k)
                    if(!broad_free(bmin, bmax, e->obs + 6 * e->ent[k])) return 0;
            }
    return 1;
}

float ko_separation(const float* obs, uint32_t n, const float bmin[3], const float bmax[3])
{
    float best = INFINITY;
    for(uint32_t o = 0; o < n; ++o) {
        const float* b = obs + 6 * o;
        float s = -INFINITY;
        for(int d = 0; d < 3; ++d) {
            float a = b[d] - bmax[d], c = bmin[d] - b[3 + d];
            if(a > s) s = a;
            if(c > s) s = c;
        }
        if(fabsf(s) < fabsf(best)) best = s;
    }
    return best;
}

/* ---------------------------------------------------------------- propagation --------- */

int ko_controls(const kpax_config* cfg, const float* u, float* ctrl_row, int32_t* steps)
{
    int N = cfg->max_propagation_duration;
    /* statePropagatorSpatialHash.cu:77 — 1 + (int)(u * N); u == 1 gives N + 1 */
    if(steps) *steps = cfg->fixed_steps ? N : 1 + f2i(u[4] * (float)N);
    float c[4] = {0, 0, 0, 0};
    for(int i = 0; i < cfg->control_dim; ++i) {
        float rng = cfg->ctrl_max[i] - cfg->ctrl_min[i];
        c[i] = cfg->ctrl_min[i] + u[i] * rng;
    }
    if(cfg->model == KPAX_MODEL_DUBINS_AIRPLANE) {
        /* drawn (a, yawRate, pitchRate), stored (yawRate, pitchRate, a): :141-144, :223-225 */
        ctrl_row[0] = c[1], ctrl_row[1] = c[2], ctrl_row[2] = c[0];
    } else {
        for(int i = 0; i < cfg->control_dim; ++i) ctrl_row[i] = c[i];
    }
    return 0;
}

typedef struct seg_ctx {
    const kpax_config* cfg;
    const ko_env* env;
    ko_seg_diag* diag;
} seg_ctx;

static void note_margin(seg_ctx* s, float value, float bound)
{
    if(s->diag) s->diag->margin = minf_(s->diag->margin, fabsf(value - bound));
}

static int all_finite(const float* x, int n)
{
    for(int i = 0; i < n; ++i)
        if(!isfinite(x[i])) return 0;
    return 1;
}

/* Box of the step's endpoints (statePropagatorSpatialHash.cu:113-125) and the grid query. */
static int step_free(seg_ctx* s, const float* p0, const float* p1)
{
    float bmin[3], bmax[3];
    for(int d = 0; d < 3; ++d) {
        if(p0[d] > p1[d]) bmin[d] = p1[d], bmax[d] = p0[d];
        else bmin[d] = p0[d], bmax[d] = p1[d];
    }
    if(s->diag && s->env) s->diag->margin = minf_(s->diag->margin, fabsf(ko_separation(s->env->obs, s->env->n, bmin, bmax)));
    return s->env ? ko_collide_hash(s->env, bmin, bmax) : 1;
}

static int fail(seg_ctx* s, int kind)
{
    if(s->diag) {
        s->diag->fail_kind = kind;
        if(kind == 4) s->diag->nonfinite = 1;
    }
    return 0;
}

/* Double integrator, statePropagatorSpatialHash.cu:72-134 (the reference's update x += h(5v + 2ah)/6, not textbook RK4). */
static int prop_di(seg_ctx* s, const float* x0, const float* c, int steps, float* x1, int* done)
{
    const float h = s->cfg->step_size, vmin = s->cfg->v_min, vmax = s->cfg->v_max, W = s->cfg->w_size;
    float ax = c[0], ay = c[1], az = c[2];
    float x = x0[0], y = x0[1], z = x0[2], vx = x0[3], vy = x0[4], vz = x0[5];
    int valid = 1, i;
    for(i = 0; i < steps; ++i) {
        float p0[3] = {x, y, z};
        x += (vx + (vx + 2 * (vx + ax * h / 2) + (vx + ax * h))) * h / 6;
        y += (vy + (vy + 2 * (vy + ay * h / 2) + (vy + ay * h))) * h / 6;
        z += (vz + (vz + 2 * (vz + az * h / 2) + (vz + az * h))) * h / 6;
        vx += (ax + 2 * ax + 2 * ax + ax) * h / 6;
        vy += (ay + 2 * ay + 2 * ay + ay) * h / 6;
        vz += (az + 2 * az + 2 * az + az) * h / 6;
        float v3[3] = {vx, vy, vz}, q3[3] = {x, y, z};
        for(int d = 0; d < 3; ++d) note_margin(s, v3[d], vmin), note_margin(s, v3[d], vmax);
        if(vx < vmin || vx > vmax || vy < vmin || vy > vmax || vz < vmin || vz > vmax) { valid = fail(s, 1); break; }
        for(int d = 0; d < 3; ++d) note_margin(s, q3[d], 0.0f), note_margin(s, q3[d], W);
        if(x < 0 || x > W || y < 0 || y > W || z < 0 || z > W) { valid = fail(s, 2); break; }
        float st[6] = {x, y, z, vx, vy, vz};
        if(!all_finite(st, 6)) { valid = fail(s, 4); break; }
        if(!step_free(s, p0, q3)) { valid = fail(s, 3); break; }
    }
    *done = i < steps ? i + 1 : steps;
    x1[0] = x, x1[1] = y, x1[2] = z, x1[3] = vx, x1[4] = vy, x1[5] = vz;
    return valid;
}

/* Dubins airplane, statePropagatorSpatialHash.cu:139-229. c = (a, yawRate, pitchRate). */
static int prop_dubins(seg_ctx* s, const float* x0, const float* c, int steps, float* x1, int* done)
{
    const kpax_config* cfg = s->cfg;
    const float h = cfg->step_size, h6 = h / 6.0f, hh = 0.5f * h;
    const float vmin = cfg->v_min, vmax = cfg->v_max, W = cfg->w_size;
    const float a = c[0], yr = c[1], pr = c[2];
    float x = x0[0], y = x0[1], z = x0[2], yaw = x0[3], pitch = x0[4], v = x0[5];
    int valid = 1, i;
    for(i = 0; i < steps; ++i) {
        float p0[3] = {x, y, z};
        x += h6 * (v * cosf(pitch) * cosf(yaw) +
                   2.0f * ((v + hh * a) * cosf(pitch + hh * pr) * cosf(yaw + hh * yr) +
                           (v + hh * a) * cosf(pitch + hh * pr) * cosf(yaw + hh * yr)) +
                   (v + h * a) * cosf(pitch + h * pr) * cosf(yaw + h * yr));
        y += h6 * (v * cosf(pitch) * sinf(yaw) +
                   2.0f * ((v + hh * a) * cosf(pitch + hh * pr) * sinf(yaw + hh * yr) +
                           (v + hh * a) * cosf(pitch + hh * pr) * sinf(yaw + hh * yr)) +
                   (v + h * a) * cosf(pitch + h * pr) * sinf(yaw + h * yr));
        z += h6 * (v * sinf(pitch) + 2.0f * ((v + hh * a) * sinf(pitch + hh * pr) + (v + hh * a) * sinf(pitch + hh * pr)) +
                   (v + h * a) * sinf(pitch + h * pr));
        yaw += h * yr;
        pitch += h * pr;
        v += h6 * (a + 2.0f * (a + a) + a);
        note_margin(s, v, vmin), note_margin(s, v, vmax);
        if(v < vmin || v > vmax) { valid = fail(s, 1); break; }
        note_margin(s, pitch, (float)cfg->pitch_min), note_margin(s, pitch, (float)cfg->pitch_max);
        /* the pitch limits are double literals (config.h:280-281): compare in double */
        if((double)pitch < cfg->pitch_min || (double)pitch > cfg->pitch_max) { valid = fail(s, 1); break; }
        float q3[3] = {x, y, z};
        for(int d = 0; d < 3; ++d) note_margin(s, q3[d], 0.0f), note_margin(s, q3[d], W);
        if(x < 0 || x > W || y < 0 || y > W || z < 0 || z > W) { valid = fail(s, 2); break; }
        float st[6] = {x, y, z, yaw, pitch, v};
        if(!all_finite(st, 6)) { valid = fail(s, 4); break; }
        if(!step_free(s, p0, q3)) { valid = fail(s, 3); break; }
    }
    *done = i < steps ? i + 1 : steps;
    x1[0] = x, x1[1] = y, x1[2] = z, x1[3] = yaw, x1[4] = pitch, x1[5] = v;
    return valid;
}

/* Quadrotor right-hand side, statePropagator.cu:325-370 (NU 10e-3, MU 2e-6, IX 1, IY 1, IZ 2,
 * GRAVITY -9.81, MASS 1: config.h:300-308). */
static void quad_ode(float* xd, const float* x0, const float* hk, float Zc, float Lc, float Mc, float Nc, float delta)
{
    const float NU = 10e-3f, MU = 2e-6f, IX = 1.0f, IY = 1.0f, IZ = 2.0f, G = -9.81f, MASS = 1.0f;
    float phi = x0[3] + delta * (hk ? hk[3] : 0);
    float theta = x0[4] + delta * (hk ? hk[4] : 0);
    float psi = x0[5] + delta * (hk ? hk[5] : 0);
    float u = x0[6] + delta * (hk ? hk[6] : 0);
    float v = x0[7] + delta * (hk ? hk[7] : 0);
    float w = x0[8] + delta * (hk ? hk[8] : 0);
    float p = x0[9] + delta * (hk ? hk[9] : 0);
    float q = x0[10] + delta * (hk ? hk[10] : 0);
    float r = x0[11] + delta * (hk ? hk[11] : 0);
    xd[0] = cosf(theta) * cosf(psi) * u + (sinf(phi) * sinf(theta) * cosf(psi) - cosf(phi) * sinf(psi)) * v +
            (cosf(phi) * sinf(theta) * cosf(psi) + sinf(phi) * sinf(psi)) * w;
    xd[1] = cosf(theta) * sinf(psi) * u + (sinf(phi) * sinf(theta) * sinf(psi) + cosf(phi) * cosf(psi)) * v +
            (cosf(phi) * sinf(theta) * sinf(psi) - sinf(phi) * cosf(psi)) * w;
    xd[2] = -sinf(theta) * u + sinf(phi) * cosf(theta) * v + cosf(phi) * cosf(theta) * w;
    xd[3] = p + (q * sinf(phi) + r * cosf(phi)) * tanf(theta);
    xd[4] = q * cosf(phi) - r * sinf(phi);
    xd[5] = (q * sinf(phi) + r * cosf(phi)) / cosf(theta);
    float XYZ = -NU * sqrtf(u * u + v * v + w * w);
    xd[6] = (r * v - q * w) - G * sinf(theta) + 1.0f / MASS * XYZ * u;
    xd[7] = (p * w - r * u) + G * cosf(theta) * sinf(phi) + 1.0f / MASS * XYZ * v;
    xd[8] = (q * u - p * v) + G * cosf(theta) * cosf(phi) + 1.0f / MASS * XYZ * w + 1.0f / MASS * Zc;
    float LMN = -MU * sqrtf(p * p + q * q + r * r);
    xd[9] = (IY - IZ) / IX * q * r + (1 / IX) * LMN * p + (1 / IX) * Lc;
    xd[10] = (IZ - IX) / IY * p * r + (1 / IY) * LMN * q + (1 / IY) * Mc;
    xd[11] = (IX - IY) / IZ * p * q + (1 / IZ) * LMN * r + (1 / IZ) * Nc;
}

/* Quadrotor RK4 loop, statePropagatorSpatialHash.cu:234-308. */
static int prop_quad(seg_ctx* s, const float* x0, const float* c, int steps, float* x1, int* done)
{
    const kpax_config* cfg = s->cfg;
    const float h = cfg->step_size, h6 = h / 6.0f, hh = 0.5f * h;
    const float vmin = cfg->v_min, vmax = cfg->v_max, wmin = cfg->w_min, wmax = cfg->w_max;
    float h0[12], k1[12], k2[12], k3[12], k4[12];
    memcpy(h0, x0, sizeof(h0));
    int valid = 1, i;
    for(i = 0; i < steps; ++i) {
        float p0[3] = {h0[0], h0[1], h0[2]};
        quad_ode(k1, h0, NULL, c[0], c[1], c[2], c[3], 1.0f);
        quad_ode(k2, h0, k1, c[0], c[1], c[2], c[3], hh);
        quad_ode(k3, h0, k2, c[0], c[1], c[2], c[3], hh);
        quad_ode(k4, h0, k3, c[0], c[1], c[2], c[3], h);
        for(int j = 0; j < 12; ++j) h0[j] += h6 * (k1[j] + 2.0f * k2[j] + 2.0f * k3[j] + k4[j]);
        for(int d = 6; d < 9; ++d) note_margin(s, h0[d], vmin), note_margin(s, h0[d], vmax);
        if(h0[6] < vmin || h0[6] > vmax || h0[7] < vmin || h0[7] > vmax || h0[8] < vmin || h0[8] > vmax) {
            valid = fail(s, 1);
            break;
        }
        for(int d = 0; d < 3; ++d) note_margin(s, h0[d], wmin), note_margin(s, h0[d], wmax);
        if(h0[0] < wmin || h0[0] > wmax || h0[1] < wmin || h0[1] > wmax || h0[2] < wmin || h0[2] > wmax) {
            valid = fail(s, 2);
            break;
        }
        if(!all_finite(h0, 12)) { valid = fail(s, 4); break; }
        if(!step_free(s, p0, h0)) { valid = fail(s, 3); break; }
    }
    *done = i < steps ? i + 1 : steps;
    memcpy(x1, h0, sizeof(h0));
    return valid;
}

int ko_propagate(const kpax_config* cfg, const ko_env* env, const float* x0, const float* u, float* row,
                 int32_t* steps_done, ko_seg_diag* diag)
{
    seg_ctx s = {cfg, env, diag};
    if(diag) diag->margin = INFINITY, diag->nonfinite = 0, diag->fail_kind = 0;
    int steps = 0, done = 0, valid = 0;
    float c[4] = {0, 0, 0, 0}, ctrl_row[4];
    ko_controls(cfg, u, ctrl_row, &steps);
    for(int i = 0; i < cfg->control_dim; ++i) c[i] = cfg->ctrl_min[i] + u[i] * (cfg->ctrl_max[i] - cfg->ctrl_min[i]);
    const int sd = cfg->state_dim;
    switch(cfg->model) {
        case KPAX_MODEL_DOUBLE_INTEGRATOR: valid = prop_di(&s, x0, c, steps, row, &done); break;
        case KPAX_MODEL_DUBINS_AIRPLANE: valid = prop_dubins(&s, x0, c, steps, row, &done); break;
        case KPAX_MODEL_QUADROTOR: valid = prop_quad(&s, x0, c, steps, row, &done); break;
        default: return 0;
    }
    for(int i = 0; i < cfg->control_dim; ++i) row[sd + i] = ctrl_row[i];
    row[sd + cfg->control_dim] = cfg->step_size * steps; /* STEP_SIZE * propagationDuration */
    if(steps_done) *steps_done = done;
    return valid;
}

void ko_propagate_batch(const kpax_config* cfg, const ko_env* env, const float* parents, const float* draws,
                        uint32_t stream, uint32_t n, float* rows, uint8_t* valid, int32_t* steps, ko_seg_diag* diag,
                        int nthreads)
{
    const int sd = cfg->state_dim, S = sd + cfg->control_dim + 1;
#pragma omp parallel for num_threads(nthreads > 0 ? nthreads : 1) schedule(dynamic, 64)
    for(long i = 0; i < (long)n; ++i) {
        float u[6];
        if(draws) memcpy(u, draws + 6 * i, sizeof(u));
        else ko_child_draws(cfg->seed, stream, 0, (uint32_t)i, u);
        int32_t done = 0;
        int ok = ko_propagate(cfg, env, parents + (size_t)sd * i, u, rows + (size_t)S * i, &done, diag ? diag + i : NULL);
        if(valid) valid[i] = (uint8_t)ok;
        if(steps) steps[i] = done;
    }
}

/* ---------------------------------------------------------------- FP64 integration ---- */

static void quad_ode_d(double* xd, const double* x0, const double* hk, const float* c, double delta)
{
    const double NU = 10e-3, MU = 2e-6, IX = 1.0, IY = 1.0, IZ = 2.0, G = -9.81;
    double s[12];
    for(int j = 3; j < 12; ++j) s[j] = x0[j] + delta * (hk ? hk[j] : 0.0);
    double phi = s[3], th = s[4], psi = s[5], u = s[6], v = s[7], w = s[8], p = s[9], q = s[10], r = s[11];
    xd[0] = cos(th) * cos(psi) * u + (sin(phi) * sin(th) * cos(psi) - cos(phi) * sin(psi)) * v +
            (cos(phi) * sin(th) * cos(psi) + sin(phi) * sin(psi)) * w;
    xd[1] = cos(th) * sin(psi) * u + (sin(phi) * sin(th) * sin(psi) + cos(phi) * cos(psi)) * v +
            (cos(phi) * sin(th) * sin(psi) - sin(phi) * cos(psi)) * w;
    xd[2] = -sin(th) * u + sin(phi) * cos(th) * v + cos(phi) * cos(th) * w;
    xd[3] = p + (q * sin(phi) + r * cos(phi)) * tan(th);
    xd[4] = q * cos(phi) - r * sin(phi);
    xd[5] = (q * sin(phi) + r * cos(phi)) / cos(th);
    double XYZ = -NU * sqrt(u * u + v * v + w * w);
    xd[6] = (r * v - q * w) - G * sin(th) + XYZ * u;
    xd[7] = (p * w - r * u) + G * cos(th) * sin(phi) + XYZ * v;
    xd[8] = (q * u - p * v) + G * cos(th) * cos(phi) + XYZ * w + (double)c[0];
    double LMN = -MU * sqrt(p * p + q * q + r * r);
    xd[9] = (IY - IZ) / IX * q * r + LMN * p / IX + (double)c[1] / IX;
    xd[10] = (IZ - IX) / IY * p * r + LMN * q / IY + (double)c[2] / IY;
    xd[11] = (IX - IY) / IZ * p * q + LMN * r / IZ + (double)c[3] / IZ;
}

void ko_integrate_f64(const kpax_config* cfg, const double* x0, const float* ctrl, int steps, int mode, double* out)
{
    const double h = (double)cfg->step_size;
    const int sd = cfg->state_dim;
    double s[12];
    memcpy(s, x0, sizeof(double) * sd);
    if(cfg->model == KPAX_MODEL_DOUBLE_INTEGRATOR) {
        for(int i = 0; i < steps; ++i)
            for(int d = 0; d < 3; ++d) {
                double a = ctrl[d], v = s[3 + d];
                if(mode == 0) s[d] += (v + (v + 2 * (v + a * h / 2) + (v + a * h))) * h / 6;
                else s[d] += h * v + 0.5 * a * h * h;
                s[3 + d] += a * h;
            }
    } else if(cfg->model == KPAX_MODEL_DUBINS_AIRPLANE) {
        /* ctrl in row layout (yawRate, pitchRate, a); the discrete map is classical RK4 */
        const double yr = ctrl[0], pr = ctrl[1], a = ctrl[2], hh = 0.5 * h;
        for(int i = 0; i < steps; ++i) {
            double yaw = s[3], pit = s[4], v = s[5];
            double vm = v + hh * a, ve = v + h * a;
            s[0] += h / 6 * (v * cos(pit) * cos(yaw) + 4 * vm * cos(pit + hh * pr) * cos(yaw + hh * yr) +
                             ve * cos(pit + h * pr) * cos(yaw + h * yr));
            s[1] += h / 6 * (v * cos(pit) * sin(yaw) + 4 * vm * cos(pit + hh * pr) * sin(yaw + hh * yr) +
                             ve * cos(pit + h * pr) * sin(yaw + h * yr));
            s[2] += h / 6 * (v * sin(pit) + 4 * vm * sin(pit + hh * pr) + ve * sin(pit + h * pr));
            s[3] += h * yr;
            s[4] += h * pr;
            s[5] += h * a;
        }
    } else {
        double k1[12], k2[12], k3[12], k4[12];
        for(int i = 0; i < steps; ++i) {
            quad_ode_d(k1, s, NULL, ctrl, 0.0);
            quad_ode_d(k2, s, k1, ctrl, 0.5 * h);
            quad_ode_d(k3, s, k2, ctrl, 0.5 * h);
            quad_ode_d(k4, s, k3, ctrl, h);
            for(int j = 0; j < 12; ++j) s[j] += h / 6 * (k1[j] + 2 * k2[j] + 2 * k3[j] + k4[j]);
        }
    }
    memcpy(out, s, sizeof(double) * sd);
}

/* ---------------------------------------------------------------- regions ------------- */

int ko_table_cols(const kpax_config* cfg) { return 3 + cfg->c_dim + cfg->v_dim; }

/* R1 min-corner table.  region_compat = 1 restates initializeRegions_kernel (Graph.cu:53-97),
 * whose id decomposition (w fastest, C_R1^2 attitude cells) differs from getRegion's (w slowest). */
void ko_region_table(const kpax_config* cfg, float* table)
{
    uint32_t n1, P;
    ko_sizes(cfg, &n1, &P, NULL);
    const int W = cfg->w_r1_length, C = cfg->c_r1_length, V = cfg->v_r1_length, cd = cfg->c_dim, vd = cfg->v_dim;
    const int cols = ko_table_cols(cfg);
    const float w_size = (cfg->w_max - cfg->w_min) / W, v_size = (cfg->v_max - cfg->v_min) / V;
    const double c_size = (cfg->c_max - cfg->c_min) / C;
    const int mulA = ipow(V, vd), mulW = ipow(C, cd) * mulA;
    for(uint32_t r = 0; r < n1; ++r) {
        float* m = table + (size_t)r * cols;
        int wi[3], ai[8], vi[8];
        if(cfg->region_compat) {
            int t = (int)r % (W * W * W);
            for(int i = 2; i >= 0; --i) wi[i] = t % W, t /= W;
            t = ((int)r / (W * W * W)) % (C * C);
            for(int i = cd - 1; i >= 0; --i) ai[i] = t % C, t /= C;
            t = ((int)r / (W * W * W * C * C)) % V;
            for(int i = vd - 1; i >= 0; --i) vi[i] = t % V, t /= V;
        } else {
            int w = (int)r / mulW, rem = (int)r % mulW, a = rem / mulA, v = rem % mulA;
            for(int i = 2; i >= 0; --i) wi[i] = w % W, w /= W;
            for(int i = cd - 1; i >= 0; --i) ai[i] = a % C, a /= C;
            for(int i = vd - 1; i >= 0; --i) vi[i] = v % V, v /= V;
        }
        for(int i = 0; i < 3; ++i) m[i] = cfg->w_min + wi[i] * w_size;
        for(int i = 0; i < cd; ++i) m[3 + i] = (float)(cfg->c_min + ai[i] * c_size);
        for(int i = 0; i < vd; ++i) m[3 + cd + i] = cfg->v_min + vi[i] * v_size;
    }
}

/* getRegion, Graph.cu:99-153.  Workspace and velocity parts in float, attitude part in double
 * (C_MIN/C_MAX are double literals). */
int ko_region_r1(const kpax_config* cfg, const float* x)
{
    const int W = cfg->w_r1_length, C = cfg->c_r1_length, V = cfg->v_r1_length, cd = cfg->c_dim, vd = cfg->v_dim;
    int w = 0, f = 1;
    for(int i = 2; i >= 0; --i) {
        int idx = clampi(f2i((float)W * (x[i] - cfg->w_min) / (cfg->w_max - cfg->w_min)), 0, W - 1);
        w += f * idx;
        f *= W;
    }
    if(vd == 1 && cd == 1) return w;
    int a = 0, v = 0;
    if(C > 1) {
        f = 1;
        for(int i = cd - 1; i >= 0; --i) {
            int idx = clampi(d2i((double)C * ((double)x[3 + i] - cfg->c_min) / (cfg->c_max - cfg->c_min)), 0, C - 1);
            a += f * idx;
            f *= C;
        }
    }
    if(V > 1) {
        f = 1;
        for(int i = vd - 1; i >= 0; --i) {
            int idx = clampi(f2i((float)V * (x[3 + cd + i] - cfg->v_min) / (cfg->v_max - cfg->v_min)), 0, V - 1);
            v += f * idx;
            f *= V;
        }
    }
    return w * ipow(C, cd) * ipow(V, vd) + a * ipow(V, vd) + v;
}

/* getSubRegion, Graph.cu:155-205. */
int ko_region_r2(const kpax_config* cfg, const float* table, const float* x, int r1)
{
    const int W2 = cfg->w_r2_length, C2 = cfg->c_r2_length, V2 = cfg->v_r2_length, cd = cfg->c_dim, vd = cfg->v_dim;
    const float* m = table + (size_t)r1 * ko_table_cols(cfg);
    const float w_size = (cfg->w_max - cfg->w_min) / cfg->w_r1_length;
    const float v_size = (cfg->v_max - cfg->v_min) / cfg->v_r1_length;
    const double c_size = (cfg->c_max - cfg->c_min) / cfg->c_r1_length;
    uint32_t P;
    ko_sizes(cfg, NULL, &P, NULL);
    int w = 0, f = 1;
    for(int i = 2; i >= 0; --i) {
        int idx = clampi(f2i((float)W2 * (x[i] - m[i]) / w_size), 0, W2 - 1);
        w += f * idx;
        f *= W2;
    }
    int a = 0, v = 0;
    if(C2 > 1) {
        f = 1;
        for(int i = cd - 1; i >= 0; --i) {
            float t = (float)C2 * (x[3 + i] - m[3 + i]);
            int idx = clampi(d2i((double)t / c_size), 0, C2 - 1);
            a += f * idx;
            f *= C2;
        }
    }
    if(V2 > 1) {
        f = 1;
        for(int i = vd - 1; i >= 0; --i) {
            int idx = clampi(f2i((float)V2 * (x[3 + cd + i] - m[3 + cd + i]) / v_size), 0, V2 - 1);
            v += f * idx;
            f *= V2;
        }
    }
    return r1 * (int)P + (w * ipow(C2, cd) * ipow(V2, vd) + a * ipow(V2, vd) + v);
}

/* ---------------------------------------------------------------- scores -------------- */

static uint32_t range_popcount(const uint32_t* bits, uint64_t lo, uint64_t hi)
{
    uint32_t n = 0;
    for(uint64_t b = lo; b < hi; ++b) n += (bits[b >> 5] >> (b & 31)) & 1u;
    return n;
}

/* Syclop-style region score (Graph.cu:241-256, 319-335) and normalisation (:297-304, :349-357)
 * with the total summed in a fixed order (the reference adds with atomics): regions in groups of
 * 32 consecutive ids, each group summed by a xor butterfly (v[i] += v[i ^ d] for d = 16 .. 1),
 * group g added to partial g mod 1024 in ascending g, then a halving tree over the partials. */
void ko_scores(const kpax_config* cfg, const int32_t* counter, const int32_t* valid, const uint32_t* r2_bits, float* scores)
{
    uint32_t n1, P;
    ko_sizes(cfg, &n1, &P, NULL);
    const float eps = cfg->epsilon;
    const float ws = (cfg->w_max - cfg->w_min) / cfg->w_r1_length;
    const float vol = ws * ws * ws;
    float* raw = (float*)malloc(sizeof(float) * n1);
    float part[1024];
    for(int j = 0; j < 1024; ++j) part[j] = 0.0f;
    for(uint32_t r = 0; r < n1; ++r) {
        float sc = 0.0f;
        if(valid[r] > 0) {
            int nv = valid[r], c = counter[r];
            float cov = (float)range_popcount(r2_bits, (uint64_t)r * P, (uint64_t)(r + 1) * P) / (float)P;
            float fv = (eps + (float)nv) / (eps + (float)nv + (float)(c - nv)) * vol;
            float fv2 = fv * fv, fv4 = fv2 * fv2, cf = (float)c;
            sc = fv4 / ((1.0f + cov) * (1.0f + cf * cf));
        }
        raw[r] = sc;
    }
    for(uint32_t g = 0; 32u * g < n1; ++g) {
        float v[32], w[32];
        for(int i = 0; i < 32; ++i) v[i] = 32u * g + i < n1 ? raw[32u * g + i] : 0.0f;
        for(int d = 16; d > 0; d >>= 1) {
            for(int i = 0; i < 32; ++i) w[i] = v[i] + v[i ^ d];
            memcpy(v, w, sizeof(v));
        }
        part[g & 1023] += v[0];
    }
    for(int s = 512; s > 0; s >>= 1)
        for(int j = 0; j < s; ++j) part[j] += part[j + s];
    const float total = part[0];
    for(uint32_t r = 0; r < n1; ++r) scores[r] = valid[r] == 0 ? 1.0f : eps + raw[r] / total;
    free(raw);
}

/* fAccept = itr * EPSILON * (1 - treeAfter / MAX_TREE_SIZE)^5 (KPAX.cu:527-528), in float. */
float ko_faccept(const kpax_config* cfg, uint32_t iter, uint32_t tree_after)
{
    float a = 1.0f - (float)tree_after / (float)cfg->max_tree_size;
    float a2 = a * a, a4 = a2 * a2, a5 = a4 * a;
    return ((float)iter * cfg->epsilon) * a5;
}

/* ---------------------------------------------------------------- plan ---------------- */

static float goal_dist(const float* x, const float* g)
{
    float dx = x[0] - g[0], dy = x[1] - g[1], dz = x[2] - g[2];
    return sqrtf(dx * dx + dy * dy + dz * dz);
}

/* Children per entry k and entries taken E for R frontier entries under a children budget B > 0
 * (KPAX.cu:323-350 as the CUDA path resolves it: k = CHILDREN_PER_ENTRY, or B / R (at least 1)
 * when the entries would exceed the budget; E = min(R, B / k)). */
static void budget_split(uint64_t R, uint32_t B, uint32_t per_entry, uint32_t* k_out, uint32_t* E_out)
{
    uint32_t k = per_entry;
    if(R * k > B) {
        k = (uint32_t)(B / (R ? R : 1));
        if(k == 0) k = 1;
    }
    *k_out = k;
    *E_out = R == 0 ? 0 : (uint32_t)(R < B / k ? R : B / k);
}

/* Entry list (repeatInd, Planner.cu:68-80).  Node i owns virtual entries [a, a + rep[i]).  When
 * the R entries exceed the budget (E < R), entry j is virtual entry floor(j * R / E): E entries
 * evenly spaced over the whole frontier (the reference gives every entry at least one child
 * instead, KPAX.cu:323-336).  A node leaves the frontier when at least one of its entries is
 * taken (KPAX.cu:372). */
static void take_entries(uint8_t* rep, uint32_t tree, uint64_t R, uint32_t E, uint32_t* entry)
{
    uint64_t a = 0;
    for(uint32_t i = 0; i < tree; ++i) {
        const uint32_t cnt = rep[i];
        if(!cnt) continue;
        const uint64_t b = a + cnt;
        const uint64_t lo = (a * E + R - 1) / R, hi = (b * E + R - 1) / R;
        for(uint64_t j = lo; j < hi; ++j) entry[j] = i;
        if(lo < hi) rep[i] = 0;
        a = b;
    }
}

void ko_frontier_compact(const kpax_config* cfg, uint8_t* rep, uint32_t n, uint32_t budget, uint32_t* entries,
                         uint32_t stats[4])
{
    uint64_t R = 0;
    for(uint32_t i = 0; i < n; ++i) {  /* a pending node of a region without valid samples */
        if(rep[i] == KO_PENDING) rep[i] = 0 < cfg->sparse_valid_threshold ? (uint8_t)cfg->sparse_repeat : 1;
        R += rep[i];
    }
    uint32_t k = cfg->children_per_entry, E = 0;
    if(budget) budget_split(R, budget, cfg->children_per_entry, &k, &E);
    take_entries(rep, n, R, E, entries);
    stats[0] = (uint32_t)R, stats[1] = k, stats[2] = E, stats[3] = E * k;
}

int ko_plan(const kpax_config* cfg, const float* init, const float* goal, const float* obs, uint32_t n_obs,
            uint32_t plan_idx, uint32_t max_iters, int stop_at_goal, ko_plan_out* out)
{
    uint32_t n1, P, S;
    ko_sizes(cfg, &n1, &P, &S);
    const uint32_t cap = cfg->max_tree_size, sd = (uint32_t)cfg->state_dim;
    const uint64_t n2 = (uint64_t)n1 * P, words = (n2 + 31) / 32;
    float* rows = (float*)calloc((size_t)cap * S, sizeof(float));
    int32_t* parent = (int32_t*)malloc(sizeof(int32_t) * cap);
    float* cost = (float*)calloc(cap, sizeof(float));
    int32_t* r1 = (int32_t*)calloc(cap, sizeof(int32_t));
    uint8_t* rep = (uint8_t*)calloc(cap, 1);
    int32_t* counter = (int32_t*)calloc(n1, sizeof(int32_t));
    int32_t* valid = (int32_t*)calloc(n1, sizeof(int32_t));
    float* scores = (float*)calloc(n1, sizeof(float));
    uint32_t* cur = (uint32_t*)calloc(words, sizeof(uint32_t));
    uint32_t* nxt = (uint32_t*)calloc(words, sizeof(uint32_t));
    float* table = (float*)malloc(sizeof(float) * n1 * ko_table_cols(cfg));
    uint32_t budget_max = cfg->expansions_per_iter;
    uint32_t* entry = (uint32_t*)malloc(sizeof(uint32_t) * (budget_max ? budget_max : 1));
    float* child = (float*)malloc(sizeof(float) * S * (budget_max ? budget_max : 1));
    int32_t* child_r1 = (int32_t*)malloc(sizeof(int32_t) * (budget_max ? budget_max : 1));
    int32_t* child_r2 = (int32_t*)malloc(sizeof(int32_t) * (budget_max ? budget_max : 1));
    uint8_t* child_ok = (uint8_t*)malloc(budget_max ? budget_max : 1);
    uint8_t* child_next = (uint8_t*)malloc(budget_max ? budget_max : 1);
    ko_env* env = ko_env_create(cfg, obs, n_obs);
    ko_region_table(cfg, table);
    for(uint32_t i = 0; i < cap; ++i) parent[i] = -1;

    memcpy(rows, init, sizeof(float) * S);
    r1[0] = ko_region_r1(cfg, rows);
    rep[0] = (uint8_t)cfg->root_repeat;
    uint32_t tree = 1, goal_idx = 0, it = 0;
    int found = 0, full = 0;
    uint64_t n_exp = 0, n_valid = 0;

    for(it = 1; it <= max_iters; ++it) {
        /* frontier: resolve the repeat counts of last iteration's nodes (KPAX.cu:476-479) */
        uint64_t R = 0;
        for(uint32_t i = 0; i < tree; ++i) {
            if(rep[i] == KO_PENDING) rep[i] = valid[r1[i]] < cfg->sparse_valid_threshold ? (uint8_t)cfg->sparse_repeat : 1;
            R += rep[i];
        }
        uint32_t B = cap - tree < budget_max ? cap - tree : budget_max;
        if(B == 0) { full = 1; it -= 1; break; }
        uint32_t k, E;
        budget_split(R, B, cfg->children_per_entry, &k, &E);
        const uint32_t n = E * k;
        take_entries(rep, tree, R, E, entry);
        memcpy(nxt, cur, sizeof(uint32_t) * words);
        /* propagateFrontier_kernel1 body (KPAX.cu:381-396) with snapshot R2 reads: the children are
         * independent (their draws, parents, the R2 snapshot and last iteration's scores are fixed),
         * so they are propagated in parallel and their counter updates applied in child order */
#pragma omp parallel for schedule(dynamic, 64)
        for(long cc = 0; cc < (long)n; ++cc) {
            const uint32_t c = (uint32_t)cc;
            float u[6], x0[12];
            ko_child_draws(cfg->seed, plan_idx, it, c, u);
            memcpy(x0, rows + (size_t)entry[c / k] * S, sizeof(float) * sd);
            float* x1 = child + (size_t)c * S;
            child_ok[c] = (uint8_t)ko_propagate(cfg, env, x0, u, x1, NULL, NULL);
            child_r1[c] = ko_region_r1(cfg, x1);
            child_r2[c] = ko_region_r2(cfg, table, x1, child_r1[c]);
        }
        for(uint32_t c = 0; c < n; ++c) {
            uint32_t p = entry[c / k];
            float u[6], x0[12];
            ko_child_draws(cfg->seed, plan_idx, it, c, u);
            memcpy(x0, rows + (size_t)p * S, sizeof(float) * sd);
            float* x1 = child + (size_t)c * S;
            int ok = child_ok[c];
            int a = child_r1[c];
            int b = child_r2[c];
            counter[a] += 1;
            child_r1[c] = a;
            child_next[c] = 0;
            if(ok) {
                valid[a] += 1;
                n_valid += 1;
                int seen = (cur[(uint32_t)b >> 5] >> (b & 31)) & 1;
                if(u[5] < scores[a] || !seen) child_next[c] = 1;
                nxt[(uint32_t)b >> 5] |= 1u << (b & 31);
                if(child_next[c] && cfg->prune) { /* PruneKPAX.cu:474-492 (pruned children are not appended) */
                    float prog = (goal_dist(x0, goal) - goal_dist(x1, goal)) / cfg->prune_progress_scale + 0.5f;
                    prog = prog < 0.0f ? 0.0f : (prog > 1.0f ? 1.0f : prog);
                    float prob = cfg->prune_exploration_bias + cfg->prune_goal_bias * prog;
                    prob = prob < cfg->epsilon ? cfg->epsilon : (prob > 1.0f ? 1.0f : prob);
                    if(!(ko_prune_draw(cfg->seed, plan_idx, it, c) < prob)) child_next[c] = 0;
                }
            }
        }
        n_exp += n;
        /* append in child order (updateFrontier_kernel, KPAX.cu:458-502) */
        uint32_t added = 0;
        for(uint32_t c = 0; c < n; ++c) {
            if(!child_next[c]) continue;
            uint32_t idx = tree + added++;
            float* x1 = child + (size_t)c * S;
            memcpy(rows + (size_t)idx * S, x1, sizeof(float) * S);
            parent[idx] = (int32_t)entry[c / k];
            cost[idx] = goal_dist(x1, goal);
            r1[idx] = child_r1[c];
            rep[idx] = KO_PENDING;
            if(cost[idx] < cfg->goal_thresh && !found) found = 1, goal_idx = idx;
        }
        /* region scores (Graph::updateVertices) */
        uint32_t* t = cur;
        cur = nxt;
        nxt = t;
        ko_scores(cfg, counter, valid, cur, scores);
        /* re-activation of old nodes (KPAX.cu:505-517) */
        float fa = ko_faccept(cfg, it, tree + added);
        for(uint32_t i = 0; i < tree; ++i) {
            if(rep[i] != 0) continue;
            if(ko_reactivate_draw(cfg->seed, plan_idx, it, i) <= scores[r1[i]] + fa) rep[i] = 1;
        }
        if(out && out->iter_children) out->iter_children[it - 1] = n;
        if(out && out->iter_appended) out->iter_appended[it - 1] = added;
        tree += added;
        if(found && stop_at_goal) break;
    }
    if(it > max_iters) it = max_iters;

    if(out) {
        kpax_result* res = &out->result;
        memset(res, 0, sizeof(*res));
        res->found = found;
        res->goal_idx = goal_idx;
        res->tree_size = tree;
        res->iters = it;
        res->tree_full = full;
        res->expansions = n_exp;
        res->valid_expansions = n_valid;
        if(found) {
            int32_t node = (int32_t)goal_idx;
            uint32_t len = 0;
            float pc = 0.0f;  /* FP32, goal to root, as the planner's path walk */
            while(node != -1) {
                if(out->path) memcpy(out->path + (size_t)len * S, rows + (size_t)node * S, sizeof(float) * S);
                if(parent[node] != -1) pc += rows[(size_t)node * S + S - 1];
                len++;
                node = parent[node];
            }
            res->path_len = len;
            res->path_cost = pc;
        }
        if(out->rows) memcpy(out->rows, rows, sizeof(float) * (size_t)tree * S);
        if(out->parents) memcpy(out->parents, parent, sizeof(int32_t) * tree);
        if(out->costs) memcpy(out->costs, cost, sizeof(float) * tree);
        if(out->r1) memcpy(out->r1, r1, sizeof(int32_t) * tree);
        if(out->repeat) memcpy(out->repeat, rep, tree);
        if(out->counter) memcpy(out->counter, counter, sizeof(int32_t) * n1);
        if(out->valid) memcpy(out->valid, valid, sizeof(int32_t) * n1);
        if(out->scores) memcpy(out->scores, scores, sizeof(float) * n1);
        if(out->r2_bits) memcpy(out->r2_bits, cur, sizeof(uint32_t) * words);
    }
    free(rows), free(parent), free(cost), free(r1), free(rep), free(counter), free(valid), free(scores);
    free(cur), free(nxt), free(table), free(entry), free(child), free(child_r1), free(child_r2), free(child_ok), free(child_next);
    ko_env_destroy(env);
    return found;
}

/* ---------------------------------------------------------------- ReKinoLite ---------- */
/* ReKinoLite (src/ReKino/ReKinoLite.cu:251-459) with the build's deterministic choices: Philox
 * draws (sample j of warp w at iteration it: child draws of index 512 w + j; the warp's epsilon /
 * choice / backtrack uniforms: counter (w, it, 2, plan)), the winner is the smallest (iteration,
 * warp), a full 200-node path restarts from the start state.  Warps are simulated one after the
 * other; a warp stops at iterations past the best goal iteration found so far, as on the GPU.
 * Returns 1 when a goal was reached: out_path holds the winner's path (start first), *out_len its
 * last index, *out_warp / *out_iter the winner. */
int ko_rekino(const kpax_config* cfg, const float* init, const float* goal, const float* obs, uint32_t n_obs,
              uint32_t num_warps, uint32_t spt, float eps, uint32_t max_iter, uint32_t plan_idx,
              float* out_path, int32_t* out_len, int32_t* out_warp, int32_t* out_iter)
{
    const uint32_t S = (uint32_t)(cfg->state_dim + cfg->control_dim + 1), sd = (uint32_t)cfg->state_dim;
    const uint32_t ns = 32u * spt, max_path = 200;
    float* path = (float*)malloc(sizeof(float) * max_path * S);
    float* cand = (float*)malloc(sizeof(float) * ns * S);
    float* dist = (float*)malloc(sizeof(float) * ns);
    ko_env* env = ko_env_create(cfg, obs, n_obs);
    uint32_t best_it = 0xFFFFFFFFu;
    int32_t best_w = -1;
    uint32_t key[2] = {(uint32_t)cfg->seed, (uint32_t)(cfg->seed >> 32)};
    for(uint32_t w = 0; w < num_warps; ++w) {
        memcpy(path, init, sizeof(float) * S);
        int depth = 0;
        for(uint32_t it = 0; it < max_iter; ++it) {
            if(best_it != 0xFFFFFFFFu && it > best_it) break;
            float x0[12];
            memcpy(x0, path + (size_t)depth * S, sizeof(float) * sd);
            for(uint32_t j = 0; j < ns; ++j) {
                float u[6];
                ko_child_draws(cfg->seed, plan_idx, it, w * 512u + j, u);
                const int ok = ko_propagate(cfg, env, x0, u, cand + (size_t)j * S, NULL, NULL);
                dist[j] = ok ? goal_dist(cand + (size_t)j * S, goal) : INFINITY;
            }
            float bd = INFINITY;
            int bj = -1;
            for(uint32_t j = 0; j < ns; ++j)
                if(dist[j] < bd) bd = dist[j], bj = (int)j;
            uint32_t c[4] = {w, it, 2u, plan_idx}, r[4];
            ko_philox4x32_10(c, key, r);
            if(eps > 0.0f && ko_u01(r[0]) < eps) {
                int total = 0;
                for(uint32_t j = 0; j < ns; ++j) total += dist[j] < INFINITY;
                if(total > 0) {
                    const int pick = (int)(ko_u01(r[1]) * (float)total);
                    int cnt = 0;
                    for(uint32_t j = 0; j < ns; ++j)
                        if(dist[j] < INFINITY) {
                            if(cnt == pick) {
                                bj = (int)j, bd = dist[j];
                                break;
                            }
                            ++cnt;
                        }
                }
            }
            if(bj >= 0) {
                if(depth + 1 >= (int)max_path) {
                    depth = 0;
                } else {
                    ++depth;
                    memcpy(path + (size_t)depth * S, cand + (size_t)bj * S, sizeof(float) * S);
                    if(bd < cfg->goal_thresh) {
                        if(it < best_it || (it == best_it && (int32_t)w < best_w)) {
                            best_it = it, best_w = (int32_t)w;
                            memcpy(out_path, path, sizeof(float) * (size_t)(depth + 1) * S);
                            *out_len = depth;
                        }
                        break;
                    }
                }
            } else if(depth > 0) {
                int back = 1 + (int)(ko_u01(r[2]) * 5.0f);
                depth = depth - back < 0 ? 0 : depth - back;
            }
        }
    }
    ko_env_destroy(env);
    free(path), free(cand), free(dist);
    *out_warp = best_w;
    *out_iter = best_w >= 0 ? (int32_t)best_it : -1;
    return best_w >= 0;
}
