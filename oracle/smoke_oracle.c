/*
 * smoke_oracle.c -- CPU restatement of the diff-solver smoke step, its JVP and
 * its VJP.  TEST INFRASTRUCTURE ONLY: this file is the checker that the CUDA
 * product is compared against.  It is never linked into the product library
 * and nothing in the product path calls it.
 *
 * The same source is compiled twice (see oracle/Makefile):
 *   REAL=float  -> libsmoke_oracle_f32.so  (operation order of the reference's
 *                                           FP32 kernels, used to pin this
 *                                           restatement against them)
 *   REAL=double -> libsmoke_oracle_f64.so  (the FP64 oracle every product field
 *                                           reports its error against)
 * Adjoint arrays are FP64 in both builds, as in the reference's adjoint views
 * (solvers/smoke/cuda_types.h:81-129).
 *
 * Every function cites the reference line it restates; paths are relative to
 * the diff-solver project root.  Functions marked "extension" have no
 * reference counterpart (inflow "set" sources, Jacobi-PCG, adjoint PCG).
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL double
#endif
typedef REAL real;
typedef double adj;

#define EXPORT __attribute__((visibility("default")))
#ifdef _OPENMP
#include <omp.h>
#define OMP_FOR _Pragma("omp parallel for schedule(static)")
#else
#define OMP_FOR
#endif

/* ------------------------------------------------------------------------ */
/* public structs (mirrored by ctypes in tests/oracle_binding.py)            */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint32_t nx, ny, nz;
    double cell_size, time_step;
} og_grid;

typedef struct {
    uint32_t modes[6];
    double values[6];
} og_sbnd;

typedef struct {
    uint32_t modes[6];
    double values[18];
} og_vbnd;

typedef struct {
    double center[3];
    double radius;
    double density;
    double temperature;
} og_inflow;

typedef struct {
    og_grid grid;
    og_vbnd velocity_boundary;
    og_sbnd pressure_boundary;
    og_sbnd density_boundary;
    og_sbnd temperature_boundary;
    uint32_t pressure_anchor;
    uint32_t vorticity_enabled;
    uint32_t solver;          /* 0: red-black Gauss-Seidel, fixed count; 1: Jacobi-PCG */
    uint32_t iterations;      /* RBGS sweeps, or PCG iteration cap */
    double tolerance;         /* PCG relative residual */
    uint32_t inflow_count;
    const og_inflow* inflows; /* extension: cells inside are set, not sourced */
    const uint32_t* cell_mask;            /* N, NULL = every cell fluid */
    const real* collider_velocity[3];     /* faces per axis, NULL = zero */
    const real* collider_density;         /* N, NULL = zero */
    const real* collider_temperature;     /* N, NULL = zero */
    const real* pressure_guess;           /* extension: start of the forward PCG solve, NULL = zero */
} og_config;

typedef struct { real* density; real* temperature; real* velocity[3]; } og_state;
typedef struct { real* density_source; real* temperature_source; real* acceleration[3]; } og_control;
typedef struct { real ambient_temperature, density_buoyancy, temperature_buoyancy, vorticity_confinement; } og_params;
typedef struct {
    real* sourced_density;
    real* sourced_temperature;
    real* force[3];
    real* centered_velocity[3];
    real* vorticity[3];
    real* magnitude;
    real* normal[3];
    real* normalizer;
    real* forced_velocity[3];
    real* advected_velocity[3];
} og_cache;
typedef struct { adj* density; adj* temperature; adj* velocity[3]; } og_state_adj;
typedef struct { adj* density_source; adj* temperature_source; adj* acceleration[3]; } og_control_adj;
typedef struct { adj ambient_temperature, density_buoyancy, temperature_buoyancy, vorticity_confinement; } og_params_adj;
typedef struct { real* density; real* temperature; real* velocity[3]; } og_state_tan;
typedef struct { real* density_source; real* temperature_source; real* acceleration[3]; } og_control_tan;

typedef struct {
    uint32_t iterations;
    double initial_residual;  /* ||b||_2 */
    double final_residual;    /* ||b - A p||_2 / ||b||_2, recomputed in FP64 */
    uint32_t converged;
} og_solve_stats;

/* ------------------------------------------------------------------------ */
/* internal grid and boundary types (operators.cu:32-113)                    */
/* ------------------------------------------------------------------------ */

typedef struct { int nx, ny, nz; real h, dt; } G;
typedef struct { uint32_t modes[6]; real values[6]; } SB;
typedef struct { uint32_t modes[6]; real values[18]; } VB;
typedef struct { real x, y, z; } V3;
typedef struct { real value; V3 gradient; } Sample;
typedef struct { V3 position; V3 derivative; } Trace;

static G to_grid(const og_grid* g) {
    G r = {(int)g->nx, (int)g->ny, (int)g->nz, (real)g->cell_size, (real)g->time_step};
    return r;
}
static SB to_sb(const og_sbnd* b) {
    SB r; for (int i = 0; i < 6; ++i) { r.modes[i] = b->modes[i]; r.values[i] = (real)b->values[i]; } return r;
}
static VB to_vb(const og_vbnd* b) {
    VB r; for (int i = 0; i < 6; ++i) r.modes[i] = b->modes[i];
    for (int i = 0; i < 18; ++i) r.values[i] = (real)b->values[i];
    return r;
}

/* operators.cu:32-34 */
static size_t cells(G g) { return (size_t)g.nx * g.ny * g.nz; }
/* operators.cu:36-39 */
static int extent(G g, int axis, int dim) {
    int base = dim == 0 ? g.nx : dim == 1 ? g.ny : g.nz;
    return base + (axis == dim ? 1 : 0);
}
/* operators.cu:41-43 */
static size_t faces(G g, int axis) { return (size_t)extent(g, axis, 0) * extent(g, axis, 1) * extent(g, axis, 2); }
/* operators.cu:45-47 */
static size_t idx3(int x, int y, int z, int nx, int ny) { return (size_t)x + (size_t)nx * ((size_t)y + (size_t)ny * (size_t)z); }
/* operators.cu:49-54 */
static void decode(size_t i, int nx, int ny, int* x, int* y, int* z) {
    *x = (int)(i % (size_t)nx); size_t yz = i / (size_t)nx; *y = (int)(yz % (size_t)ny); *z = (int)(yz / (size_t)ny);
}
/* operators.cu:80-86 */
static int vperiodic(const VB* b, int d) { return b->modes[2 * d] == 3u && b->modes[2 * d + 1] == 3u; }
static int speriodic(const SB* b, int d) { return b->modes[2 * d] == 2u && b->modes[2 * d + 1] == 2u; }
/* operators.cu:88-96 */
static int wrapi(int v, int p) { int r = v % p; return r < 0 ? r + p : r; }
static int clampi(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static int map_coord(int v, int size, int per, int period) { return per ? wrapi(v, period) : clampi(v, 0, size - 1); }
static int mask_at(const uint32_t* m, size_t i) { return m ? m[i] != 0u : 0; }
static real rfloor(real v) { return (real)floor((double)v); }
static real rmin(real a, real b) { return a < b ? a : b; }
static real rmax(real a, real b) { return a > b ? a : b; }

/* operators.cu:98-103 */
static size_t mapped_cell(int x, int y, int z, G g, int px, int py, int pz) {
    x = map_coord(x, g.nx, px, g.nx); y = map_coord(y, g.ny, py, g.ny); z = map_coord(z, g.nz, pz, g.nz);
    return idx3(x, y, z, g.nx, g.ny);
}
/* operators.cu:105-113 */
static size_t mapped_face(int x, int y, int z, G g, int axis, const VB* b) {
    int ex = extent(g, axis, 0), ey = extent(g, axis, 1), ez = extent(g, axis, 2);
    x = map_coord(x, ex, vperiodic(b, 0), g.nx); y = map_coord(y, ey, vperiodic(b, 1), g.ny); z = map_coord(z, ez, vperiodic(b, 2), g.nz);
    return idx3(x, y, z, ex, ey);
}
/* operators.cu:115-123 */
/* The reference compares the int coordinate with the grid's uint32_t
 * extent (cuda_types.h:13-19), so `x >= grid.nx` is also true for x < 0:
 * below the grid, an upper face with a fixed value is hit too (after the
 * lower face's own test).  Restated with unsigned comparisons. */
static int beyond(int c, int n) { return (unsigned)c >= (unsigned)n; }
/* max(0, min(n - 1, c)) with one uint32_t operand: an unsigned clamp, so
 * c = -1 maps to n - 1 (used by solid_at and the vorticity stencils). */
static int uclamp(int c, int n) { unsigned u = (unsigned)c, m = (unsigned)(n - 1); return (int)(u < m ? u : m); }
static real load_scalar(const real* v, int x, int y, int z, G g, const SB* b) {
    if (x < 0 && b->modes[0] == 0u) return b->values[0];
    if (beyond(x, g.nx) && b->modes[1] == 0u) return b->values[1];
    if (y < 0 && b->modes[2] == 0u) return b->values[2];
    if (beyond(y, g.ny) && b->modes[3] == 0u) return b->values[3];
    if (z < 0 && b->modes[4] == 0u) return b->values[4];
    if (beyond(z, g.nz) && b->modes[5] == 0u) return b->values[5];
    return v[mapped_cell(x, y, z, g, speriodic(b, 0), speriodic(b, 1), speriodic(b, 2))];
}
/* operators.cu:125-134 */
static real load_face(const real* v, int axis, int x, int y, int z, G g, const VB* b) {
    int c[3] = {x, y, z};
    for (int d = 0; d < 3; ++d) {
        int size = extent(g, axis, d);
        if (c[d] >= 0 && c[d] < size) continue;
        int face = 2 * d + (c[d] >= size);
        if (b->modes[face] == 0u || (b->modes[face] == 2u && axis == d)) return b->values[3 * face + axis];
    }
    return v[mapped_face(x, y, z, g, axis, b)];
}
/* trilinear value + gradient of an 8-value cell (operators.cu:150-163, 180-193) */
static Sample trilinear(real v8[2][2][2], real tx, real ty, real tz, real h) {
    real wx[2] = {(real)1 - tx, tx}, wy[2] = {(real)1 - ty, ty}, wz[2] = {(real)1 - tz, tz};
    Sample s; s.value = 0; s.gradient.x = s.gradient.y = s.gradient.z = 0;
    for (int dz = 0; dz < 2; ++dz) {
        for (int dy = 0; dy < 2; ++dy) {
            for (int dx = 0; dx < 2; ++dx) s.value += wx[dx] * wy[dy] * wz[dz] * v8[dz][dy][dx];
            s.gradient.x += wy[dy] * wz[dz] * (v8[dz][dy][1] - v8[dz][dy][0]) / h;
        }
        for (int dx = 0; dx < 2; ++dx) s.gradient.y += wx[dx] * wz[dz] * (v8[dz][1][dx] - v8[dz][0][dx]) / h;
    }
    for (int dy = 0; dy < 2; ++dy)
        for (int dx = 0; dx < 2; ++dx) s.gradient.z += wx[dx] * wy[dy] * (v8[1][dy][dx] - v8[0][dy][dx]) / h;
    return s;
}
/* operators.cu:136-164 */
static Sample sample_scalar(const real* v, V3 p, G g, const SB* b) {
    real gx = p.x / g.h - (real)0.5, gy = p.y / g.h - (real)0.5, gz = p.z / g.h - (real)0.5;
    int x0 = (int)rfloor(gx), y0 = (int)rfloor(gy), z0 = (int)rfloor(gz);
    real v8[2][2][2];
    for (int dz = 0; dz < 2; ++dz) for (int dy = 0; dy < 2; ++dy) for (int dx = 0; dx < 2; ++dx)
        v8[dz][dy][dx] = load_scalar(v, x0 + dx, y0 + dy, z0 + dz, g, b);
    return trilinear(v8, gx - (real)x0, gy - (real)y0, gz - (real)z0, g.h);
}
/* operators.cu:166-194 */
static Sample sample_face(const real* v, int axis, V3 p, G g, const VB* b) {
    real gx = p.x / g.h - (axis == 0 ? (real)0 : (real)0.5);
    real gy = p.y / g.h - (axis == 1 ? (real)0 : (real)0.5);
    real gz = p.z / g.h - (axis == 2 ? (real)0 : (real)0.5);
    int x0 = (int)rfloor(gx), y0 = (int)rfloor(gy), z0 = (int)rfloor(gz);
    real v8[2][2][2];
    for (int dz = 0; dz < 2; ++dz) for (int dy = 0; dy < 2; ++dy) for (int dx = 0; dx < 2; ++dx)
        v8[dz][dy][dx] = load_face(v, axis, x0 + dx, y0 + dy, z0 + dz, g, b);
    return trilinear(v8, gx - (real)x0, gy - (real)y0, gz - (real)z0, g.h);
}
/* operators.cu:196-215 */
static void scatter_scalar(adj* v, V3 p, adj a, G g, const SB* b) {
    real gx = p.x / g.h - (real)0.5, gy = p.y / g.h - (real)0.5, gz = p.z / g.h - (real)0.5;
    int x0 = (int)rfloor(gx), y0 = (int)rfloor(gy), z0 = (int)rfloor(gz);
    adj wx[2] = {1.0 - (adj)(gx - (real)x0), (adj)(gx - (real)x0)};
    adj wy[2] = {1.0 - (adj)(gy - (real)y0), (adj)(gy - (real)y0)};
    adj wz[2] = {1.0 - (adj)(gz - (real)z0), (adj)(gz - (real)z0)};
    for (int dz = 0; dz < 2; ++dz) for (int dy = 0; dy < 2; ++dy) for (int dx = 0; dx < 2; ++dx) {
        int x = x0 + dx, y = y0 + dy, z = z0 + dz;
        if ((x < 0 && b->modes[0] == 0u) || (beyond(x, g.nx) && b->modes[1] == 0u) || (y < 0 && b->modes[2] == 0u) ||
            (beyond(y, g.ny) && b->modes[3] == 0u) || (z < 0 && b->modes[4] == 0u) || (beyond(z, g.nz) && b->modes[5] == 0u)) continue;
        v[mapped_cell(x, y, z, g, speriodic(b, 0), speriodic(b, 1), speriodic(b, 2))] += a * wx[dx] * wy[dy] * wz[dz];
    }
}
/* operators.cu:217-240 */
static void scatter_face(adj* v, int axis, V3 p, adj a, G g, const VB* b) {
    real gx = p.x / g.h - (axis == 0 ? (real)0 : (real)0.5);
    real gy = p.y / g.h - (axis == 1 ? (real)0 : (real)0.5);
    real gz = p.z / g.h - (axis == 2 ? (real)0 : (real)0.5);
    int x0 = (int)rfloor(gx), y0 = (int)rfloor(gy), z0 = (int)rfloor(gz);
    adj wx[2] = {1.0 - (adj)(gx - (real)x0), (adj)(gx - (real)x0)};
    adj wy[2] = {1.0 - (adj)(gy - (real)y0), (adj)(gy - (real)y0)};
    adj wz[2] = {1.0 - (adj)(gz - (real)z0), (adj)(gz - (real)z0)};
    for (int dz = 0; dz < 2; ++dz) for (int dy = 0; dy < 2; ++dy) for (int dx = 0; dx < 2; ++dx) {
        int c[3] = {x0 + dx, y0 + dy, z0 + dz};
        int constant = 0;
        for (int d = 0; d < 3; ++d) {
            int size = extent(g, axis, d);
            if (c[d] >= 0 && c[d] < size) continue;
            int face = 2 * d + (c[d] >= size);
            if (b->modes[face] == 0u || (b->modes[face] == 2u && axis == d)) constant = 1;
        }
        if (!constant) v[mapped_face(c[0], c[1], c[2], g, axis, b)] += a * wx[dx] * wy[dy] * wz[dz];
    }
}
/* operators.cu:242-244 */
static V3 sample_velocity(real* const u[3], V3 p, G g, const VB* b) {
    V3 r = {sample_face(u[0], 0, p, g, b).value, sample_face(u[1], 1, p, g, b).value, sample_face(u[2], 2, p, g, b).value};
    return r;
}
/* operators.cu:246-254 */
static int solid_at(V3 p, const uint32_t* mask, G g, const VB* b) {
    if (!mask) return 0;
    if (vperiodic(b, 0)) p.x -= rfloor(p.x / ((real)g.nx * g.h)) * (real)g.nx * g.h;
    if (vperiodic(b, 1)) p.y -= rfloor(p.y / ((real)g.ny * g.h)) * (real)g.ny * g.h;
    if (vperiodic(b, 2)) p.z -= rfloor(p.z / ((real)g.nz * g.h)) * (real)g.nz * g.h;
    int x = uclamp((int)rfloor(p.x / g.h), g.nx);
    int y = uclamp((int)rfloor(p.y / g.h), g.ny);
    int z = uclamp((int)rfloor(p.z / g.h), g.nz);
    return mask[idx3(x, y, z, g.nx, g.ny)] != 0u;
}
/* operators.cu:256-276 */
static Trace trace_rk2(V3 s, real* const u[3], const uint32_t* mask, G g, const VB* b) {
    V3 v0 = sample_velocity(u, s, g, b);
    V3 mid = {s.x - (real)0.5 * g.dt * v0.x, s.y - (real)0.5 * g.dt * v0.y, s.z - (real)0.5 * g.dt * v0.z};
    V3 v1 = sample_velocity(u, mid, g, b);
    V3 raw = {s.x - g.dt * v1.x, s.y - g.dt * v1.y, s.z - g.dt * v1.z};
    V3 der = {1, 1, 1};
    V3 mx = {(real)g.nx * g.h, (real)g.ny * g.h, (real)g.nz * g.h};
    if (!vperiodic(b, 0) && (raw.x < 0 || raw.x > mx.x)) { raw.x = rmin(rmax(raw.x, 0), mx.x); der.x = 0; }
    if (!vperiodic(b, 1) && (raw.y < 0 || raw.y > mx.y)) { raw.y = rmin(rmax(raw.y, 0), mx.y); der.y = 0; }
    if (!vperiodic(b, 2) && (raw.z < 0 || raw.z > mx.z)) { raw.z = rmin(rmax(raw.z, 0), mx.z); der.z = 0; }
    Trace t;
    if (!solid_at(raw, mask, g, b)) { t.position = raw; t.derivative = der; return t; }
    real lo = 0, hi = 1;
    for (int it = 0; it < 8; ++it) {
        real f = (real)0.5 * (lo + hi);
        V3 test = {s.x + f * (raw.x - s.x), s.y + f * (raw.y - s.y), s.z + f * (raw.z - s.z)};
        if (solid_at(test, mask, g, b)) hi = f; else lo = f;
    }
    t.position.x = s.x + lo * (raw.x - s.x); t.position.y = s.y + lo * (raw.y - s.y); t.position.z = s.z + lo * (raw.z - s.z);
    t.derivative.x = lo * der.x; t.derivative.y = lo * der.y; t.derivative.z = lo * der.z;
    return t;
}
/* operators.cu:278-284 */
static V3 face_position(int axis, int x, int y, int z, G g) {
    V3 p = {((real)x + (axis == 0 ? (real)0 : (real)0.5)) * g.h, ((real)y + (axis == 1 ? (real)0 : (real)0.5)) * g.h, ((real)z + (axis == 2 ? (real)0 : (real)0.5)) * g.h};
    return p;
}
static V3 cell_position(int x, int y, int z, G g) {
    V3 p = {((real)x + (real)0.5) * g.h, ((real)y + (real)0.5) * g.h, ((real)z + (real)0.5) * g.h};
    return p;
}

/* ------------------------------------------------------------------------ */
/* inflow (extension): a cell whose centre lies inside a sphere is set to the */
/* sphere's value instead of being sourced.                                   */
/* ------------------------------------------------------------------------ */
static int inflow_hit(const og_config* c, G g, size_t i, real* dens, real* temp) {
    if (c->inflow_count == 0) return 0;
    int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
    V3 p = cell_position(x, y, z, g);
    int hit = 0;
    for (uint32_t k = 0; k < c->inflow_count; ++k) {
        const og_inflow* f = &c->inflows[k];
        real dx = p.x - (real)f->center[0], dy = p.y - (real)f->center[1], dz = p.z - (real)f->center[2];
        real r = (real)f->radius;
        if (dx * dx + dy * dy + dz * dz <= r * r) { hit = 1; *dens = (real)f->density; *temp = (real)f->temperature; }
    }
    return hit;
}

/* ------------------------------------------------------------------------ */
/* forward kernels                                                           */
/* ------------------------------------------------------------------------ */

/* operators.cu:286-290 (+ inflow extension: which = 0 density, 1 temperature) */
static void source_forward(const og_config* c, G g, const real* state, const real* src, real* out, int which) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        real d, t;
        if (mask_at(c->cell_mask, i)) { out[i] = 0; continue; }
        if (inflow_hit(c, g, i, &d, &t)) { out[i] = which == 0 ? d : t; continue; }
        out[i] = state[i] + g.dt * src[i];
    }
}
/* operators.cu:575-577 (+ inflow: set cells carry no tangent) */
static void source_jvp(const og_config* c, G g, const real* st, const real* sr, real* out) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        real d, t;
        if (mask_at(c->cell_mask, i) || inflow_hit(c, g, i, &d, &t)) { out[i] = 0; continue; }
        out[i] = st[i] + g.dt * sr[i];
    }
}
/* operators.cu:297-302 (+ inflow: set cells pass no adjoint) */
static void source_vjp(const og_config* c, G g, const adj* oa, adj* sa, adj* ra) {
    for (size_t i = 0; i < cells(g); ++i) {
        real d, t;
        if (mask_at(c->cell_mask, i) || inflow_hit(c, g, i, &d, &t)) continue;
        sa[i] += oa[i];
        ra[i] += (adj)g.dt * oa[i];
    }
}
/* operators.cu:304-313 */
static void buoyancy_forward(const og_config* c, G g, const real* rho, const real* T, real* const ext[3], const og_params* pr, real* f[3]) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i)) { f[0][i] = f[1][i] = f[2][i] = 0; continue; }
        f[0][i] = ext[0][i];
        f[1][i] = ext[1][i] + pr->density_buoyancy * rho[i] + pr->temperature_buoyancy * (T[i] - pr->ambient_temperature);
        f[2][i] = ext[2][i];
    }
}
/* operators.cu:315-324 */
static void buoyancy_jvp(const og_config* c, G g, const real* rho, const real* T, const real* rt, const real* Tt, real* const et[3],
                         const og_params* pr, const og_params* pt, real* f[3]) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i)) { f[0][i] = f[1][i] = f[2][i] = 0; continue; }
        f[0][i] = et[0][i];
        f[1][i] = et[1][i] + pr->density_buoyancy * rt[i] + pt->density_buoyancy * rho[i] +
                  pr->temperature_buoyancy * (Tt[i] - pt->ambient_temperature) + pt->temperature_buoyancy * (T[i] - pr->ambient_temperature);
        f[2][i] = et[2][i];
    }
}
/* operators.cu:326-337 */
static void buoyancy_vjp(const og_config* c, G g, const real* rho, const real* T, const og_params* pr, adj* const fa[3],
                         adj* ra, adj* Ta, adj* ea[3], og_params_adj* pa) {
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i)) continue;
        ea[0][i] += fa[0][i]; ea[1][i] += fa[1][i]; ea[2][i] += fa[2][i];
        ra[i] += (adj)pr->density_buoyancy * fa[1][i];
        Ta[i] += (adj)pr->temperature_buoyancy * fa[1][i];
        pa->ambient_temperature += -(adj)pr->temperature_buoyancy * fa[1][i];
        pa->density_buoyancy += (adj)rho[i] * fa[1][i];
        pa->temperature_buoyancy += (adj)(T[i] - pr->ambient_temperature) * fa[1][i];
    }
}
static int in_grid(G g, int x, int y, int z) { return x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz; }
/* operators.cu:339-356 */
static real averaged_force(const real* f, int axis, int x, int y, int z, G g, const uint32_t* m) {
    int fx = x - (axis == 0), fy = y - (axis == 1), fz = z - (axis == 2);
    real sum = 0, count = 0;
    if (in_grid(g, fx, fy, fz)) { size_t c = idx3(fx, fy, fz, g.nx, g.ny); if (!mask_at(m, c)) { sum += f[c]; count += 1; } }
    if (in_grid(g, x, y, z)) { size_t c = idx3(x, y, z, g.nx, g.ny); if (!mask_at(m, c)) { sum += f[c]; count += 1; } }
    return count == 0 ? (real)0 : sum / count;
}
/* operators.cu:358-364, 599-602 */
static void integrate(const og_config* c, G g, real* const u[3], real* const f[3], real* out[3]) {
    for (int a = 0; a < 3; ++a)
        OMP_FOR
        for (size_t i = 0; i < faces(g, a); ++i) {
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            out[a][i] = u[a][i] + g.dt * averaged_force(f[a], a, x, y, z, g, c->cell_mask);
        }
}
/* operators.cu:366-379, 608-611 */
static void integrate_vjp(const og_config* c, G g, adj* const oa[3], adj* ua[3], adj* fa[3]) {
    for (int a = 0; a < 3; ++a)
        for (size_t i = 0; i < faces(g, a); ++i) {
            ua[a][i] += oa[a][i];
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            int cs[2][3] = {{x - (a == 0), y - (a == 1), z - (a == 2)}, {x, y, z}};
            int count = 0;
            for (int s = 0; s < 2; ++s)
                if (in_grid(g, cs[s][0], cs[s][1], cs[s][2]) && !mask_at(c->cell_mask, idx3(cs[s][0], cs[s][1], cs[s][2], g.nx, g.ny))) ++count;
            if (count == 0) continue;
            for (int s = 0; s < 2; ++s)
                if (in_grid(g, cs[s][0], cs[s][1], cs[s][2]) && !mask_at(c->cell_mask, idx3(cs[s][0], cs[s][1], cs[s][2], g.nx, g.ny)))
                    fa[a][idx3(cs[s][0], cs[s][1], cs[s][2], g.nx, g.ny)] += (adj)g.dt * oa[a][i] / count;
        }
}
/* operators.cu:381-388, 613-616 */
static void advect_velocity(const og_config* c, G g, const VB* b, real* const u[3], real* out[3]) {
    for (int a = 0; a < 3; ++a)
        OMP_FOR
        for (size_t i = 0; i < faces(g, a); ++i) {
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            Trace t = trace_rk2(face_position(a, x, y, z, g), u, c->cell_mask, g, b);
            out[a][i] = sample_face(u[a], a, t.position, g, b).value;
        }
}
static VB zero_values_v(const VB* b) { VB r = *b; for (int i = 0; i < 18; ++i) r.values[i] = 0; return r; }
static SB zero_values_s(const SB* b) { SB r = *b; for (int i = 0; i < 6; ++i) r.values[i] = 0; return r; }
/* operators.cu:390-413, 618-621 */
static void advect_velocity_jvp(const og_config* c, G g, const VB* b, real* const u[3], real* const ut[3], real* out[3]) {
    VB tb = zero_values_v(b);
    for (int a = 0; a < 3; ++a)
        OMP_FOR
        for (size_t i = 0; i < faces(g, a); ++i) {
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            V3 s = face_position(a, x, y, z, g);
            V3 v0 = sample_velocity(u, s, g, b);
            V3 t0 = sample_velocity(ut, s, g, &tb);
            V3 mid = {s.x - (real)0.5 * g.dt * v0.x, s.y - (real)0.5 * g.dt * v0.y, s.z - (real)0.5 * g.dt * v0.z};
            V3 midt = {-(real)0.5 * g.dt * t0.x, -(real)0.5 * g.dt * t0.y, -(real)0.5 * g.dt * t0.z};
            Sample vs[3] = {sample_face(u[0], 0, mid, g, b), sample_face(u[1], 1, mid, g, b), sample_face(u[2], 2, mid, g, b)};
            V3 st = sample_velocity(ut, mid, g, &tb);
            V3 v1t = {st.x + vs[0].gradient.x * midt.x + vs[0].gradient.y * midt.y + vs[0].gradient.z * midt.z,
                      st.y + vs[1].gradient.x * midt.x + vs[1].gradient.y * midt.y + vs[1].gradient.z * midt.z,
                      st.z + vs[2].gradient.x * midt.x + vs[2].gradient.y * midt.y + vs[2].gradient.z * midt.z};
            Trace t = trace_rk2(s, u, c->cell_mask, g, b);
            V3 pt = {-t.derivative.x * g.dt * v1t.x, -t.derivative.y * g.dt * v1t.y, -t.derivative.z * g.dt * v1t.z};
            Sample src = sample_face(u[a], a, t.position, g, b);
            out[a][i] = sample_face(ut[a], a, t.position, g, &tb).value + src.gradient.x * pt.x + src.gradient.y * pt.y + src.gradient.z * pt.z;
        }
}
/* operators.cu:415-439, 623-626 */
static void advect_velocity_vjp(const og_config* c, G g, const VB* b, real* const u[3], adj* const oa[3], adj* ua[3]) {
    for (int a = 0; a < 3; ++a)
        for (size_t i = 0; i < faces(g, a); ++i) {
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            V3 s = face_position(a, x, y, z, g);
            V3 v0 = sample_velocity(u, s, g, b);
            V3 mid = {s.x - (real)0.5 * g.dt * v0.x, s.y - (real)0.5 * g.dt * v0.y, s.z - (real)0.5 * g.dt * v0.z};
            Trace t = trace_rk2(s, u, c->cell_mask, g, b);
            Sample src = sample_face(u[a], a, t.position, g, b);
            adj o = oa[a][i];
            scatter_face(ua[a], a, t.position, o, g, b);
            adj v1x = -(adj)(t.derivative.x * g.dt * src.gradient.x) * o;
            adj v1y = -(adj)(t.derivative.y * g.dt * src.gradient.y) * o;
            adj v1z = -(adj)(t.derivative.z * g.dt * src.gradient.z) * o;
            Sample ms[3] = {sample_face(u[0], 0, mid, g, b), sample_face(u[1], 1, mid, g, b), sample_face(u[2], 2, mid, g, b)};
            scatter_face(ua[0], 0, mid, v1x, g, b);
            scatter_face(ua[1], 1, mid, v1y, g, b);
            scatter_face(ua[2], 2, mid, v1z, g, b);
            adj mx = ms[0].gradient.x * v1x + ms[1].gradient.x * v1y + ms[2].gradient.x * v1z;
            adj my = ms[0].gradient.y * v1x + ms[1].gradient.y * v1y + ms[2].gradient.y * v1z;
            adj mz = ms[0].gradient.z * v1x + ms[1].gradient.z * v1y + ms[2].gradient.z * v1z;
            scatter_face(ua[0], 0, s, -0.5 * (adj)g.dt * mx, g, b);
            scatter_face(ua[1], 1, s, -0.5 * (adj)g.dt * my, g, b);
            scatter_face(ua[2], 2, s, -0.5 * (adj)g.dt * mz, g, b);
        }
}
/* operators.cu:441-449 */
static int adjacent_solid(int a, int x, int y, int z, G g, const uint32_t* m) {
    if (!m) return 0;
    int f[3] = {x - (a == 0), y - (a == 1), z - (a == 2)}, s[3] = {x, y, z};
    if (in_grid(g, f[0], f[1], f[2]) && m[idx3(f[0], f[1], f[2], g.nx, g.ny)] != 0u) return 1;
    if (in_grid(g, s[0], s[1], s[2]) && m[idx3(s[0], s[1], s[2], g.nx, g.ny)] != 0u) return 1;
    return 0;
}
/* operators.cu:451-464 */
static int constrained_boundary(int a, int x, int y, int z, G g, const VB* b) {
    int coord = a == 0 ? x : a == 1 ? y : z, mx = a == 0 ? g.nx : a == 1 ? g.ny : g.nz;
    if (coord != 0 && coord != mx) return 0;
    uint32_t mode = b->modes[a * 2 + (coord == mx)];
    return mode == 0u || mode == 2u;
}
static real boundary_velocity(int a, int x, int y, int z, G g, const VB* b) {
    int coord = a == 0 ? x : a == 1 ? y : z, mx = a == 0 ? g.nx : a == 1 ? g.ny : g.nz;
    return b->values[(a * 2 + (coord == mx)) * 3 + a];
}
/* operators.cu:466-481, 628-631; collider may be NULL (constrain_velocity_jvp, :633-638) */
static void constrain(const og_config* c, G g, const VB* b, real* const col[3], real* const u[3], real* out[3]) {
    for (int a = 0; a < 3; ++a)
        OMP_FOR
        for (size_t i = 0; i < faces(g, a); ++i) {
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            if (constrained_boundary(a, x, y, z, g, b)) { out[a][i] = boundary_velocity(a, x, y, z, g, b); continue; }
            if (adjacent_solid(a, x, y, z, g, c->cell_mask)) { out[a][i] = col && col[a] ? col[a][i] : (real)0; continue; }
            if (vperiodic(b, a) && (a == 0 ? x == g.nx : a == 1 ? y == g.ny : z == g.nz)) {
                if (a == 0) x = 0;
                if (a == 1) y = 0;
                if (a == 2) z = 0;
                out[a][i] = u[a][idx3(x, y, z, extent(g, a, 0), extent(g, a, 1))];
                continue;
            }
            out[a][i] = u[a][i];
        }
}
/* operators.cu:483-497, 640-643 */
static void constrain_vjp(const og_config* c, G g, const VB* b, adj* const oa[3], adj* ua[3]) {
    for (int a = 0; a < 3; ++a)
        for (size_t i = 0; i < faces(g, a); ++i) {
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            if (constrained_boundary(a, x, y, z, g, b) || adjacent_solid(a, x, y, z, g, c->cell_mask)) continue;
            if (vperiodic(b, a) && (a == 0 ? x == g.nx : a == 1 ? y == g.ny : z == g.nz)) {
                if (a == 0) x = 0;
                if (a == 1) y = 0;
                if (a == 2) z = 0;
                ua[a][idx3(x, y, z, extent(g, a, 0), extent(g, a, 1))] += oa[a][i];
                continue;
            }
            ua[a][i] += oa[a][i];
        }
}
/* operators.cu:499-507, 645-648 */
static void advect_scalar(const og_config* c, G g, const SB* sb, const VB* vb, const real* col, const real* src, real* const u[3], real* out) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i)) { out[i] = col ? col[i] : (real)0; continue; }
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        Trace t = trace_rk2(cell_position(x, y, z, g), u, c->cell_mask, g, vb);
        out[i] = sample_scalar(src, t.position, g, sb).value;
    }
}
/* operators.cu:509-535, 650-653 */
static void advect_scalar_jvp(const og_config* c, G g, const SB* sb, const VB* vb, const real* src, const real* srct, real* const u[3], real* const ut[3], real* out) {
    SB stb = zero_values_s(sb);
    VB vtb = zero_values_v(vb);
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i)) { out[i] = 0; continue; }
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        V3 s = cell_position(x, y, z, g);
        V3 v0 = sample_velocity(u, s, g, vb);
        V3 t0 = sample_velocity(ut, s, g, &vtb);
        V3 mid = {s.x - (real)0.5 * g.dt * v0.x, s.y - (real)0.5 * g.dt * v0.y, s.z - (real)0.5 * g.dt * v0.z};
        V3 midt = {-(real)0.5 * g.dt * t0.x, -(real)0.5 * g.dt * t0.y, -(real)0.5 * g.dt * t0.z};
        Sample vs[3] = {sample_face(u[0], 0, mid, g, vb), sample_face(u[1], 1, mid, g, vb), sample_face(u[2], 2, mid, g, vb)};
        V3 st = sample_velocity(ut, mid, g, &vtb);
        V3 v1t = {st.x + vs[0].gradient.x * midt.x + vs[0].gradient.y * midt.y + vs[0].gradient.z * midt.z,
                  st.y + vs[1].gradient.x * midt.x + vs[1].gradient.y * midt.y + vs[1].gradient.z * midt.z,
                  st.z + vs[2].gradient.x * midt.x + vs[2].gradient.y * midt.y + vs[2].gradient.z * midt.z};
        Trace t = trace_rk2(s, u, c->cell_mask, g, vb);
        V3 pt = {-t.derivative.x * g.dt * v1t.x, -t.derivative.y * g.dt * v1t.y, -t.derivative.z * g.dt * v1t.z};
        Sample smp = sample_scalar(src, t.position, g, sb);
        out[i] = sample_scalar(srct, t.position, g, &stb).value + smp.gradient.x * pt.x + smp.gradient.y * pt.y + smp.gradient.z * pt.z;
    }
}
/* operators.cu:537-561, 655-658 */
static void advect_scalar_vjp(const og_config* c, G g, const SB* sb, const VB* vb, const real* src, real* const u[3], const adj* oa, adj* sa, adj* ua[3]) {
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i)) continue;
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        V3 s = cell_position(x, y, z, g);
        V3 v0 = sample_velocity(u, s, g, vb);
        V3 mid = {s.x - (real)0.5 * g.dt * v0.x, s.y - (real)0.5 * g.dt * v0.y, s.z - (real)0.5 * g.dt * v0.z};
        Trace t = trace_rk2(s, u, c->cell_mask, g, vb);
        Sample smp = sample_scalar(src, t.position, g, sb);
        adj o = oa[i];
        scatter_scalar(sa, t.position, o, g, sb);
        adj v1x = -(adj)(t.derivative.x * g.dt * smp.gradient.x) * o;
        adj v1y = -(adj)(t.derivative.y * g.dt * smp.gradient.y) * o;
        adj v1z = -(adj)(t.derivative.z * g.dt * smp.gradient.z) * o;
        Sample ms[3] = {sample_face(u[0], 0, mid, g, vb), sample_face(u[1], 1, mid, g, vb), sample_face(u[2], 2, mid, g, vb)};
        scatter_face(ua[0], 0, mid, v1x, g, vb);
        scatter_face(ua[1], 1, mid, v1y, g, vb);
        scatter_face(ua[2], 2, mid, v1z, g, vb);
        adj mx = ms[0].gradient.x * v1x + ms[1].gradient.x * v1y + ms[2].gradient.x * v1z;
        adj my = ms[0].gradient.y * v1x + ms[1].gradient.y * v1y + ms[2].gradient.y * v1z;
        adj mz = ms[0].gradient.z * v1x + ms[1].gradient.z * v1y + ms[2].gradient.z * v1z;
        scatter_face(ua[0], 0, s, -0.5 * (adj)g.dt * mx, g, vb);
        scatter_face(ua[1], 1, s, -0.5 * (adj)g.dt * my, g, vb);
        scatter_face(ua[2], 2, s, -0.5 * (adj)g.dt * mz, g, vb);
    }
}

/* ------------------------------------------------------------------------ */
/* vorticity confinement (operators.cu:660-846, 973-1002)                    */
/* ------------------------------------------------------------------------ */
static const real smooth_eps = (real)1.0e-6;

/* operators.cu:662-674 */
/* `max(0, min(grid.nx - 1, x))` in the reference mixes uint32_t and int;
 * CUDA's mixed min/max compare as unsigned, so x = -1 lands on nx - 1
 * (the far side) and x >= nx on nx - 1. */
static real cload(const real* v, int x, int y, int z, G g) {
    return v[idx3(uclamp(x, g.nx), uclamp(y, g.ny), uclamp(z, g.nz), g.nx, g.ny)];
}
static void cscatter(adj* v, int x, int y, int z, G g, adj a) {
    v[idx3(uclamp(x, g.nx), uclamp(y, g.ny), uclamp(z, g.nz), g.nx, g.ny)] += a;
}
/* operators.cu:676-685 */
static void centered_velocity(const og_config* c, G g, real* const u[3], real* cv[3]) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        if (mask_at(c->cell_mask, i)) { cv[0][i] = cv[1][i] = cv[2][i] = 0; continue; }
        cv[0][i] = (real)0.5 * (u[0][idx3(x, y, z, g.nx + 1, g.ny)] + u[0][idx3(x + 1, y, z, g.nx + 1, g.ny)]);
        cv[1][i] = (real)0.5 * (u[1][idx3(x, y, z, g.nx, g.ny + 1)] + u[1][idx3(x, y + 1, z, g.nx, g.ny + 1)]);
        cv[2][i] = (real)0.5 * (u[2][idx3(x, y, z, g.nx, g.ny)] + u[2][idx3(x, y, z + 1, g.nx, g.ny)]);
    }
}
/* operators.cu:687-701 */
static void curl_magnitude(const og_config* c, G g, real* const cv[3], real* w[3], real* mag) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        if (mask_at(c->cell_mask, i)) { w[0][i] = w[1][i] = w[2][i] = 0; mag[i] = smooth_eps; continue; }
        real is = (real)0.5 / g.h;
        real wx = (cload(cv[2], x, y + 1, z, g) - cload(cv[2], x, y - 1, z, g) - cload(cv[1], x, y, z + 1, g) + cload(cv[1], x, y, z - 1, g)) * is;
        real wy = (cload(cv[0], x, y, z + 1, g) - cload(cv[0], x, y, z - 1, g) - cload(cv[2], x + 1, y, z, g) + cload(cv[2], x - 1, y, z, g)) * is;
        real wz = (cload(cv[1], x + 1, y, z, g) - cload(cv[1], x - 1, y, z, g) - cload(cv[0], x, y + 1, z, g) + cload(cv[0], x, y - 1, z, g)) * is;
        w[0][i] = wx; w[1][i] = wy; w[2][i] = wz;
        mag[i] = (real)sqrt((double)(wx * wx + wy * wy + wz * wz + smooth_eps * smooth_eps));
    }
}
/* operators.cu:703-720 */
static void vorticity_normal(const og_config* c, G g, const real* mag, real* n[3], real* nz_) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        if (mask_at(c->cell_mask, i)) { n[0][i] = n[1][i] = n[2][i] = 0; nz_[i] = smooth_eps; continue; }
        real is = (real)0.5 / g.h;
        real gx = (cload(mag, x + 1, y, z, g) - cload(mag, x - 1, y, z, g)) * is;
        real gy = (cload(mag, x, y + 1, z, g) - cload(mag, x, y - 1, z, g)) * is;
        real gz = (cload(mag, x, y, z + 1, g) - cload(mag, x, y, z - 1, g)) * is;
        real len = (real)sqrt((double)(gx * gx + gy * gy + gz * gz + smooth_eps * smooth_eps));
        n[0][i] = gx / len; n[1][i] = gy / len; n[2][i] = gz / len; nz_[i] = len;
    }
}
/* operators.cu:722-729 */
static void add_vorticity_force(const og_config* c, G g, real* const w[3], real* const n[3], real conf, real* f[3]) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i)) continue;
        real s = conf * g.h;
        f[0][i] += s * (n[1][i] * w[2][i] - n[2][i] * w[1][i]);
        f[1][i] += s * (n[2][i] * w[0][i] - n[0][i] * w[2][i]);
        f[2][i] += s * (n[0][i] * w[1][i] - n[1][i] * w[0][i]);
    }
}
/* operators.cu:973-979 */
static void vorticity_forward(const og_config* c, G g, real* const u[3], real conf, og_cache* k, real* f[3]) {
    centered_velocity(c, g, u, k->centered_velocity);
    curl_magnitude(c, g, k->centered_velocity, k->vorticity, k->magnitude);
    vorticity_normal(c, g, k->magnitude, k->normal, k->normalizer);
    add_vorticity_force(c, g, k->vorticity, k->normal, conf, f);
}
/* operators.cu:981-988 with kernels :731-771; scratch: 3 + 3 + 1 + 3 arrays of N */
static void vorticity_jvp(const og_config* c, G g, real* const ut[3], real conf, real conft, const og_cache* k, real* ft[3], real* scratch) {
    size_t n = cells(g);
    real* cvt[3] = {scratch, scratch + n, scratch + 2 * n};
    real* wt[3] = {scratch + 3 * n, scratch + 4 * n, scratch + 5 * n};
    real* mt = scratch + 6 * n;
    real* nt[3] = {scratch + 7 * n, scratch + 8 * n, scratch + 9 * n};
    centered_velocity(c, g, ut, cvt);
    curl_magnitude(c, g, cvt, wt, mt);
    for (size_t i = 0; i < n; ++i)  /* :731-735 */
        mt[i] = !mask_at(c->cell_mask, i) ? (k->vorticity[0][i] * wt[0][i] + k->vorticity[1][i] * wt[1][i] + k->vorticity[2][i] * wt[2][i]) / k->magnitude[i] : (real)0;
    for (size_t i = 0; i < n; ++i) {  /* :737-753 */
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        if (mask_at(c->cell_mask, i)) { nt[0][i] = nt[1][i] = nt[2][i] = 0; continue; }
        real is = (real)0.5 / g.h;
        real gx = (cload(mt, x + 1, y, z, g) - cload(mt, x - 1, y, z, g)) * is;
        real gy = (cload(mt, x, y + 1, z, g) - cload(mt, x, y - 1, z, g)) * is;
        real gz = (cload(mt, x, y, z + 1, g) - cload(mt, x, y, z - 1, g)) * is;
        real pr = k->normal[0][i] * gx + k->normal[1][i] * gy + k->normal[2][i] * gz;
        nt[0][i] = (gx - k->normal[0][i] * pr) / k->normalizer[i];
        nt[1][i] = (gy - k->normal[1][i] * pr) / k->normalizer[i];
        nt[2][i] = (gz - k->normal[2][i] * pr) / k->normalizer[i];
    }
    for (size_t i = 0; i < n; ++i) {  /* :755-771 */
        if (mask_at(c->cell_mask, i)) continue;
        real* const* w = k->vorticity; real* const* nn = k->normal;
        real cx = nn[1][i] * w[2][i] - nn[2][i] * w[1][i];
        real cy = nn[2][i] * w[0][i] - nn[0][i] * w[2][i];
        real cz = nn[0][i] * w[1][i] - nn[1][i] * w[0][i];
        real tx = nt[1][i] * w[2][i] + nn[1][i] * wt[2][i] - nt[2][i] * w[1][i] - nn[2][i] * wt[1][i];
        real ty = nt[2][i] * w[0][i] + nn[2][i] * wt[0][i] - nt[0][i] * w[2][i] - nn[0][i] * wt[2][i];
        real tz = nt[0][i] * w[1][i] + nn[0][i] * wt[1][i] - nt[1][i] * w[0][i] - nn[1][i] * wt[0][i];
        ft[0][i] += g.h * (conft * cx + conf * tx);
        ft[1][i] += g.h * (conft * cy + conf * ty);
        ft[2][i] += g.h * (conft * cz + conf * tz);
    }
}
/* operators.cu:990-1002 with kernels :773-846; scratch: 10 adjoint arrays of N */
static void vorticity_vjp(const og_config* c, G g, real conf, const og_cache* k, adj* const fa[3], adj* ua[3], adj* conf_adj, adj* scratch) {
    size_t n = cells(g);
    memset(scratch, 0, 10 * n * sizeof(adj));
    adj* ca[3] = {scratch, scratch + n, scratch + 2 * n};
    adj* wa[3] = {scratch + 3 * n, scratch + 4 * n, scratch + 5 * n};
    adj* ma = scratch + 6 * n;
    adj* na[3] = {scratch + 7 * n, scratch + 8 * n, scratch + 9 * n};
    real* const* w = k->vorticity; real* const* nn = k->normal;
    for (size_t i = 0; i < n; ++i) {  /* :773-789 */
        if (mask_at(c->cell_mask, i)) continue;
        real cx = nn[1][i] * w[2][i] - nn[2][i] * w[1][i];
        real cy = nn[2][i] * w[0][i] - nn[0][i] * w[2][i];
        real cz = nn[0][i] * w[1][i] - nn[1][i] * w[0][i];
        adj s = (adj)conf * (adj)g.h;
        *conf_adj += (adj)g.h * ((adj)cx * fa[0][i] + (adj)cy * fa[1][i] + (adj)cz * fa[2][i]);
        na[0][i] += s * ((adj)w[1][i] * fa[2][i] - (adj)w[2][i] * fa[1][i]);
        na[1][i] += s * ((adj)w[2][i] * fa[0][i] - (adj)w[0][i] * fa[2][i]);
        na[2][i] += s * ((adj)w[0][i] * fa[1][i] - (adj)w[1][i] * fa[0][i]);
        wa[0][i] += s * (fa[1][i] * (adj)nn[2][i] - fa[2][i] * (adj)nn[1][i]);
        wa[1][i] += s * (fa[2][i] * (adj)nn[0][i] - fa[0][i] * (adj)nn[2][i]);
        wa[2][i] += s * (fa[0][i] * (adj)nn[1][i] - fa[1][i] * (adj)nn[0][i]);
    }
    for (size_t i = 0; i < n; ++i) {  /* :791-807 */
        if (mask_at(c->cell_mask, i)) continue;
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        adj pr = (adj)nn[0][i] * na[0][i] + (adj)nn[1][i] * na[1][i] + (adj)nn[2][i] * na[2][i];
        adj gx = (na[0][i] - (adj)nn[0][i] * pr) / (adj)k->normalizer[i];
        adj gy = (na[1][i] - (adj)nn[1][i] * pr) / (adj)k->normalizer[i];
        adj gz = (na[2][i] - (adj)nn[2][i] * pr) / (adj)k->normalizer[i];
        adj s = 0.5 / (adj)g.h;
        cscatter(ma, x + 1, y, z, g, s * gx); cscatter(ma, x - 1, y, z, g, -s * gx);
        cscatter(ma, x, y + 1, z, g, s * gy); cscatter(ma, x, y - 1, z, g, -s * gy);
        cscatter(ma, x, y, z + 1, g, s * gz); cscatter(ma, x, y, z - 1, g, -s * gz);
    }
    for (size_t i = 0; i < n; ++i) {  /* :809-816 */
        if (mask_at(c->cell_mask, i)) continue;
        adj s = ma[i] / (adj)k->magnitude[i];
        wa[0][i] += s * (adj)w[0][i]; wa[1][i] += s * (adj)w[1][i]; wa[2][i] += s * (adj)w[2][i];
    }
    for (size_t i = 0; i < n; ++i) {  /* :818-833 */
        if (mask_at(c->cell_mask, i)) continue;
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        adj s = 0.5 / (adj)g.h;
        adj ax = wa[0][i] * s, ay = wa[1][i] * s, az = wa[2][i] * s;
        cscatter(ca[2], x, y + 1, z, g, ax); cscatter(ca[2], x, y - 1, z, g, -ax);
        cscatter(ca[1], x, y, z + 1, g, -ax); cscatter(ca[1], x, y, z - 1, g, ax);
        cscatter(ca[0], x, y, z + 1, g, ay); cscatter(ca[0], x, y, z - 1, g, -ay);
        cscatter(ca[2], x + 1, y, z, g, -ay); cscatter(ca[2], x - 1, y, z, g, ay);
        cscatter(ca[1], x + 1, y, z, g, az); cscatter(ca[1], x - 1, y, z, g, -az);
        cscatter(ca[0], x, y + 1, z, g, -az); cscatter(ca[0], x, y - 1, z, g, az);
    }
    for (size_t i = 0; i < n; ++i) {  /* :835-846 */
        if (mask_at(c->cell_mask, i)) continue;
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        ua[0][idx3(x, y, z, g.nx + 1, g.ny)] += 0.5 * ca[0][i]; ua[0][idx3(x + 1, y, z, g.nx + 1, g.ny)] += 0.5 * ca[0][i];
        ua[1][idx3(x, y, z, g.nx, g.ny + 1)] += 0.5 * ca[1][i]; ua[1][idx3(x, y + 1, z, g.nx, g.ny + 1)] += 0.5 * ca[1][i];
        ua[2][idx3(x, y, z, g.nx, g.ny)] += 0.5 * ca[2][i]; ua[2][idx3(x, y, z + 1, g.nx, g.ny)] += 0.5 * ca[2][i];
    }
}

/* ------------------------------------------------------------------------ */
/* pressure (operators.cu:848-969, 1004-1031)                                */
/* ------------------------------------------------------------------------ */

/* operators.cu:852-873 */
static void pressure_neighbor(G g, const SB* b, const uint32_t* m, int x, int y, int z, int d, int dir,
                              int* nx, int* ny, int* nz, int* connected, int* fixed, real* fv) {
    *nx = x + (d == 0 ? dir : 0); *ny = y + (d == 1 ? dir : 0); *nz = z + (d == 2 ? dir : 0);
    int coord = d == 0 ? *nx : d == 1 ? *ny : *nz, size = d == 0 ? g.nx : d == 1 ? g.ny : g.nz;
    *fixed = 0; *fv = 0;
    if (coord < 0 || coord >= size) {
        if (speriodic(b, d)) {
            if (d == 0) *nx = wrapi(*nx, g.nx);
            if (d == 1) *ny = wrapi(*ny, g.ny);
            if (d == 2) *nz = wrapi(*nz, g.nz);
        } else {
            int face = d * 2 + (dir > 0);
            *fixed = b->modes[face] == 0u; *fv = b->values[face]; *connected = 0;
            return;
        }
    }
    *connected = !mask_at(m, idx3(*nx, *ny, *nz, g.nx, g.ny));
}
/* operators.cu:875-883 */
static void pressure_rhs(const og_config* c, G g, real* const u[3], real* rhs) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i) || i == (size_t)c->pressure_anchor) { rhs[i] = 0; continue; }
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        real div = (u[0][idx3(x + 1, y, z, g.nx + 1, g.ny)] - u[0][idx3(x, y, z, g.nx + 1, g.ny)] +
                    u[1][idx3(x, y + 1, z, g.nx, g.ny + 1)] - u[1][idx3(x, y, z, g.nx, g.ny + 1)] +
                    u[2][idx3(x, y, z + 1, g.nx, g.ny)] - u[2][idx3(x, y, z, g.nx, g.ny)]) / g.h;
        rhs[i] = -g.h * g.h * div / g.dt;
    }
}
/* operators.cu:885-902 */
static void rbgs_sweep(const og_config* c, G g, const SB* b, int parity, const real* rhs, real* p) {
    for (size_t i = 0; i < cells(g); ++i) {
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        if (((x + y + z) & 1) != parity || mask_at(c->cell_mask, i) || i == (size_t)c->pressure_anchor) continue;
        real sum = rhs[i], diag = 0;
        for (int d = 0; d < 3; ++d) for (int dir = -1; dir <= 1; dir += 2) {
            int nx, ny, nz, con, fix; real fv;
            pressure_neighbor(g, b, c->cell_mask, x, y, z, d, dir, &nx, &ny, &nz, &con, &fix, &fv);
            if (con) { sum += p[idx3(nx, ny, nz, g.nx, g.ny)]; diag += 1; }
            else if (fix) { sum += fv; diag += 1; }
        }
        p[i] = diag == 0 ? (real)0 : sum / diag;
    }
}
/* operators.cu:904-910 */
static int projectable(G g, int a, int x, int y, int z, const uint32_t* m, size_t* first, size_t* second) {
    int fx = x - (a == 0), fy = y - (a == 1), fz = z - (a == 2);
    if (!in_grid(g, fx, fy, fz) || !in_grid(g, x, y, z)) return 0;
    *first = idx3(fx, fy, fz, g.nx, g.ny); *second = idx3(x, y, z, g.nx, g.ny);
    return !mask_at(m, *first) && !mask_at(m, *second);
}
/* operators.cu:912-920 */
static void project_velocity(const og_config* c, G g, real* const u[3], const real* p, real* out[3]) {
    for (int a = 0; a < 3; ++a)
        OMP_FOR
        for (size_t i = 0; i < faces(g, a); ++i) {
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            size_t f, s;
            if (!projectable(g, a, x, y, z, c->cell_mask, &f, &s)) { out[a][i] = u[a][i]; continue; }
            out[a][i] = u[a][i] - g.dt * (p[s] - p[f]) / g.h;
        }
}
/* operators.cu:922-933 */
static void project_velocity_reverse(const og_config* c, G g, adj* const oa[3], adj* ua[3], adj* pa) {
    for (int a = 0; a < 3; ++a)
        for (size_t i = 0; i < faces(g, a); ++i) {
            ua[a][i] += oa[a][i];
            int x, y, z; decode(i, extent(g, a, 0), extent(g, a, 1), &x, &y, &z);
            size_t f, s;
            if (!projectable(g, a, x, y, z, c->cell_mask, &f, &s)) continue;
            adj sc = (adj)g.dt * oa[a][i] / (adj)g.h;
            pa[f] += sc; pa[s] -= sc;
        }
}
/* operators.cu:935-955 */
static void rbgs_reverse_sweep(const og_config* c, G g, const SB* b, int parity, adj* pa, adj* ra) {
    for (size_t i = 0; i < cells(g); ++i) {
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        if (((x + y + z) & 1) != parity || mask_at(c->cell_mask, i) || i == (size_t)c->pressure_anchor) continue;
        real diag = 0; size_t nb[6]; int cnt = 0;
        for (int d = 0; d < 3; ++d) for (int dir = -1; dir <= 1; dir += 2) {
            int nx, ny, nz, con, fix; real fv;
            pressure_neighbor(g, b, c->cell_mask, x, y, z, d, dir, &nx, &ny, &nz, &con, &fix, &fv);
            if (con) { nb[cnt++] = idx3(nx, ny, nz, g.nx, g.ny); diag += 1; }
            else if (fix) diag += 1;
        }
        adj a = diag == 0 ? 0.0 : pa[i] / (adj)diag;
        pa[i] = 0; ra[i] += a;
        for (int k = 0; k < cnt; ++k) pa[nb[k]] += a;
    }
}
/* operators.cu:957-969 */
static void pressure_rhs_reverse(const og_config* c, G g, const adj* ra, adj* ua[3]) {
    for (size_t i = 0; i < cells(g); ++i) {
        if (mask_at(c->cell_mask, i) || i == (size_t)c->pressure_anchor) continue;
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        adj s = -(adj)g.h * ra[i] / (adj)g.dt;
        ua[0][idx3(x + 1, y, z, g.nx + 1, g.ny)] += s; ua[0][idx3(x, y, z, g.nx + 1, g.ny)] -= s;
        ua[1][idx3(x, y + 1, z, g.nx, g.ny + 1)] += s; ua[1][idx3(x, y, z, g.nx, g.ny + 1)] -= s;
        ua[2][idx3(x, y, z + 1, g.nx, g.ny)] += s; ua[2][idx3(x, y, z, g.nx, g.ny)] -= s;
    }
}

/* ---- the linear system RBGS converges to (extension: explicit operator) ----
 * Row i (fluid, not the anchor, diagonal > 0):
 *     diag_i p_i - sum_{connected j} p_j = rhs_i + sum_{fixed faces} value
 * Every other cell holds p = 0.  This is the fixed point of rbgs_sweep. */
static int cell_active(const og_config* c, G g, const SB* b, size_t i, double* diag, double* fixed_sum) {
    if (mask_at(c->cell_mask, i) || i == (size_t)c->pressure_anchor) return 0;
    int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
    double d = 0, fs = 0;
    for (int dd = 0; dd < 3; ++dd) for (int dir = -1; dir <= 1; dir += 2) {
        int nx, ny, nz, con, fix; real fv;
        pressure_neighbor(g, b, c->cell_mask, x, y, z, dd, dir, &nx, &ny, &nz, &con, &fix, &fv);
        if (con) d += 1; else if (fix) { d += 1; fs += (double)fv; }
    }
    *diag = d; *fixed_sum = fs;
    return d > 0;
}
static void apply_operator(const og_config* c, G g, const SB* b, const double* diag, const uint8_t* active, const double* p, double* q) {
    OMP_FOR
    for (size_t i = 0; i < cells(g); ++i) {
        if (!active[i]) { q[i] = 0; continue; }
        int x, y, z; decode(i, g.nx, g.ny, &x, &y, &z);
        double s = diag[i] * p[i];
        for (int d = 0; d < 3; ++d) for (int dir = -1; dir <= 1; dir += 2) {
            int nx, ny, nz, con, fix; real fv;
            pressure_neighbor(g, b, c->cell_mask, x, y, z, d, dir, &nx, &ny, &nz, &con, &fix, &fv);
            if (con) { size_t j = idx3(nx, ny, nz, g.nx, g.ny); if (active[j]) s -= p[j]; }
        }
        q[i] = s;
    }
}
/* Jacobi-preconditioned CG in FP64 on the system above (extension).  rhs is
 * the pressure_rhs output; guess may be NULL (zero guess). */
static void pcg_solve(const og_config* c, G g, const SB* b, const real* rhs, const real* guess, uint32_t max_it, double tol,
                      real* p_out, og_solve_stats* st) {
    size_t n = cells(g);
    double* diag = calloc(n, sizeof(double));
    uint8_t* act = calloc(n, 1);
    double* bb = calloc(n, sizeof(double));
    double* x = calloc(n, sizeof(double));
    double* r = calloc(n, sizeof(double));
    double* p = calloc(n, sizeof(double));
    double* q = calloc(n, sizeof(double));
    double bnorm = 0;
    #pragma omp parallel for schedule(static) reduction(+:bnorm)
    for (size_t i = 0; i < n; ++i) {
        double fs = 0;
        act[i] = (uint8_t)cell_active(c, g, b, i, &diag[i], &fs);
        bb[i] = act[i] ? (double)rhs[i] + fs : 0.0;
        x[i] = (act[i] && guess) ? (double)guess[i] : 0.0;
        bnorm += bb[i] * bb[i];
    }
    bnorm = sqrt(bnorm);
    apply_operator(c, g, b, diag, act, x, q);
    double rz = 0, rr = 0;
    #pragma omp parallel for schedule(static) reduction(+:rz, rr)
    for (size_t i = 0; i < n; ++i) {
        r[i] = act[i] ? bb[i] - q[i] : 0.0;
        p[i] = act[i] ? r[i] / diag[i] : 0.0;
        rz += r[i] * p[i]; rr += r[i] * r[i];
    }
    uint32_t it = 0;
    int conv = bnorm == 0.0 || sqrt(rr) <= tol * bnorm;
    while (!conv && it < max_it) {
        apply_operator(c, g, b, diag, act, p, q);
        double pq = 0;
        #pragma omp parallel for schedule(static) reduction(+:pq)
        for (size_t i = 0; i < n; ++i) pq += p[i] * q[i];
        double alpha = rz / pq, rzn = 0; rr = 0;
        #pragma omp parallel for schedule(static) reduction(+:rzn, rr)
        for (size_t i = 0; i < n; ++i) {
            x[i] += alpha * p[i]; r[i] -= alpha * q[i];
            if (act[i]) { rzn += r[i] * r[i] / diag[i]; rr += r[i] * r[i]; }
        }
        double beta = rzn / rz; rz = rzn;
        #pragma omp parallel for schedule(static)
        for (size_t i = 0; i < n; ++i) p[i] = act[i] ? r[i] / diag[i] + beta * p[i] : 0.0;
        ++it;
        conv = sqrt(rr) <= tol * bnorm;
    }
    for (size_t i = 0; i < n; ++i) p_out[i] = act[i] ? (real)x[i] : (real)0;
    /* true residual of the stored (REAL) solution */
    for (size_t i = 0; i < n; ++i) x[i] = (double)p_out[i];
    apply_operator(c, g, b, diag, act, x, q);
    double tr = 0;
    #pragma omp parallel for schedule(static) reduction(+:tr)
    for (size_t i = 0; i < n; ++i) if (act[i]) tr += (bb[i] - q[i]) * (bb[i] - q[i]);
    if (st) { st->iterations = it; st->initial_residual = bnorm; st->final_residual = bnorm > 0 ? sqrt(tr) / bnorm : 0.0; st->converged = (uint32_t)conv; }
    free(diag); free(act); free(bb); free(x); free(r); free(p); free(q);
}
/* relative residual ||b - A p|| / ||b|| of a given pressure (FP64) */
static double relative_residual(const og_config* c, G g, const SB* b, const real* rhs, const real* pin) {
    size_t n = cells(g);
    double* diag = calloc(n, sizeof(double)); uint8_t* act = calloc(n, 1);
    double* x = calloc(n, sizeof(double)); double* q = calloc(n, sizeof(double)); double* bb = calloc(n, sizeof(double));
    double bn = 0;
    for (size_t i = 0; i < n; ++i) { double fs = 0; act[i] = (uint8_t)cell_active(c, g, b, i, &diag[i], &fs); bb[i] = act[i] ? (double)rhs[i] + fs : 0; x[i] = act[i] ? (double)pin[i] : 0; bn += bb[i] * bb[i]; }
    apply_operator(c, g, b, diag, act, x, q);
    double tr = 0;
    for (size_t i = 0; i < n; ++i) if (act[i]) tr += (bb[i] - q[i]) * (bb[i] - q[i]);
    free(diag); free(act); free(x); free(q); free(bb);
    return bn > 0 ? sqrt(tr / bn) : 0.0;
}
/* Adjoint of the converged solve (extension): solves A^T lambda_b = lambda_p
 * with A symmetric, in FP64, and adds lambda_b to rhs_adj on active cells. */
static void adjoint_solve(const og_config* c, G g, const SB* b, const adj* pa, uint32_t max_it, double tol, adj* ra, og_solve_stats* st) {
    size_t n = cells(g);
    real* rhs = calloc(n, sizeof(real));
    real* sol = calloc(n, sizeof(real));
    /* The adjoint right-hand side is FP64; solve it in FP64 through a
     * zero-boundary copy of the problem so fixed values do not enter. */
    double* diag = calloc(n, sizeof(double)); uint8_t* act = calloc(n, 1);
    double *x = calloc(n, sizeof(double)), *r = calloc(n, sizeof(double)), *p = calloc(n, sizeof(double)), *q = calloc(n, sizeof(double));
    double bn = 0;
    for (size_t i = 0; i < n; ++i) { double fs; act[i] = (uint8_t)cell_active(c, g, b, i, &diag[i], &fs); r[i] = act[i] ? pa[i] : 0; bn += r[i] * r[i]; }
    bn = sqrt(bn);
    double rz = 0, rr = 0;
    for (size_t i = 0; i < n; ++i) { p[i] = act[i] ? r[i] / diag[i] : 0; rz += r[i] * p[i]; rr += r[i] * r[i]; }
    uint32_t it = 0; int conv = bn == 0.0 || sqrt(rr) <= tol * bn;
    while (!conv && it < max_it) {
        apply_operator(c, g, b, diag, act, p, q);
        double pq = 0; for (size_t i = 0; i < n; ++i) pq += p[i] * q[i];
        double al = rz / pq, rzn = 0; rr = 0;
        for (size_t i = 0; i < n; ++i) { x[i] += al * p[i]; r[i] -= al * q[i]; if (act[i]) { rzn += r[i] * r[i] / diag[i]; rr += r[i] * r[i]; } }
        double be = rzn / rz; rz = rzn;
        for (size_t i = 0; i < n; ++i) p[i] = act[i] ? r[i] / diag[i] + be * p[i] : 0;
        ++it; conv = sqrt(rr) <= tol * bn;
    }
    for (size_t i = 0; i < n; ++i) if (act[i]) ra[i] += x[i];
    if (st) { st->iterations = it; st->initial_residual = bn; st->final_residual = bn > 0 ? sqrt(rr) / bn : 0; st->converged = (uint32_t)conv; }
    free(rhs); free(sol); free(diag); free(act); free(x); free(r); free(p); free(q);
}

/* operators.cu:1004-1013; solver 0 = the reference's RBGS, 1 = Jacobi-PCG */
static void projection_forward(const og_config* c, G g, const SB* pb, real* const u[3], real* p, real* rhs, real* out[3], og_solve_stats* st) {
    memset(p, 0, cells(g) * sizeof(real));
    pressure_rhs(c, g, u, rhs);
    if (c->solver == 0) {
        for (uint32_t it = 0; it < c->iterations; ++it) { rbgs_sweep(c, g, pb, 0, rhs, p); rbgs_sweep(c, g, pb, 1, rhs, p); }
        if (st) { st->iterations = c->iterations; st->initial_residual = 0; st->final_residual = relative_residual(c, g, pb, rhs, p); st->converged = 1; }
    } else {
        pcg_solve(c, g, pb, rhs, c->pressure_guess, c->iterations, c->tolerance, p, st);
    }
    project_velocity(c, g, u, p, out);
}
/* operators.cu:1020-1031; solver 1 replaces the reversed sweeps by the adjoint solve */
static void projection_vjp(const og_config* c, G g, const SB* pb, adj* const oa[3], adj* pa, adj* ra, adj* ua[3], og_solve_stats* st) {
    size_t n = cells(g);
    memset(pa, 0, n * sizeof(adj)); memset(ra, 0, n * sizeof(adj));
    project_velocity_reverse(c, g, oa, ua, pa);
    if (c->solver == 0) {
        for (uint32_t it = 0; it < c->iterations; ++it) { rbgs_reverse_sweep(c, g, pb, 1, pa, ra); rbgs_reverse_sweep(c, g, pb, 0, pa, ra); }
    } else {
        adjoint_solve(c, g, pb, pa, c->iterations, c->tolerance, ra, st);
    }
    pressure_rhs_reverse(c, g, ra, ua);
}

/* ------------------------------------------------------------------------ */
/* exported kernels (for per-operator parity)                                */
/* ------------------------------------------------------------------------ */
EXPORT void og_source_forward(const og_config* c, const real* state, const real* src, real* out, int which) { source_forward(c, to_grid(&c->grid), state, src, out, which); }
EXPORT void og_buoyancy_forward(const og_config* c, const real* rho, const real* T, real* const ext[3], const og_params* pr, real* f[3]) { buoyancy_forward(c, to_grid(&c->grid), rho, T, ext, pr, f); }
EXPORT void og_integrate(const og_config* c, real* const u[3], real* const f[3], real* out[3]) { integrate(c, to_grid(&c->grid), u, f, out); }
EXPORT void og_advect_velocity(const og_config* c, real* const u[3], real* out[3]) { VB b = to_vb(&c->velocity_boundary); advect_velocity(c, to_grid(&c->grid), &b, u, out); }
EXPORT void og_constrain(const og_config* c, real* const col[3], real* const u[3], real* out[3]) { VB b = to_vb(&c->velocity_boundary); constrain(c, to_grid(&c->grid), &b, col, u, out); }
EXPORT void og_advect_scalar(const og_config* c, const og_sbnd* sb, const real* col, const real* src, real* const u[3], real* out) {
    SB s = to_sb(sb); VB v = to_vb(&c->velocity_boundary); advect_scalar(c, to_grid(&c->grid), &s, &v, col, src, u, out);
}
EXPORT void og_pressure_rhs(const og_config* c, real* const u[3], real* rhs) { pressure_rhs(c, to_grid(&c->grid), u, rhs); }
EXPORT void og_rbgs(const og_config* c, const real* rhs, real* p, uint32_t iterations) {
    SB b = to_sb(&c->pressure_boundary); G g = to_grid(&c->grid);
    for (uint32_t it = 0; it < iterations; ++it) { rbgs_sweep(c, g, &b, 0, rhs, p); rbgs_sweep(c, g, &b, 1, rhs, p); }
}
EXPORT void og_pcg(const og_config* c, const real* rhs, const real* guess, uint32_t max_it, double tol, real* p, og_solve_stats* st) {
    SB b = to_sb(&c->pressure_boundary); pcg_solve(c, to_grid(&c->grid), &b, rhs, guess, max_it, tol, p, st);
}
EXPORT double og_relative_residual(const og_config* c, const real* rhs, const real* p) {
    SB b = to_sb(&c->pressure_boundary); return relative_residual(c, to_grid(&c->grid), &b, rhs, p);
}
EXPORT void og_apply_operator(const og_config* c, const double* p, double* q) {
    G g = to_grid(&c->grid); SB b = to_sb(&c->pressure_boundary); size_t n = cells(g);
    double* diag = calloc(n, sizeof(double)); uint8_t* act = calloc(n, 1);
    for (size_t i = 0; i < n; ++i) { double fs; act[i] = (uint8_t)cell_active(c, g, &b, i, &diag[i], &fs); }
    apply_operator(c, g, &b, diag, act, p, q);
    free(diag); free(act);
}
EXPORT void og_project_velocity(const og_config* c, real* const u[3], const real* p, real* out[3]) { project_velocity(c, to_grid(&c->grid), u, p, out); }
EXPORT void og_vorticity_forward(const og_config* c, real* const u[3], real conf, og_cache* k, real* f[3]) { vorticity_forward(c, to_grid(&c->grid), u, conf, k, f); }
EXPORT void og_advect_velocity_vjp(const og_config* c, real* const u[3], adj* const oa[3], adj* ua[3]) { VB b = to_vb(&c->velocity_boundary); advect_velocity_vjp(c, to_grid(&c->grid), &b, u, oa, ua); }
EXPORT void og_advect_scalar_vjp(const og_config* c, const og_sbnd* sb, const real* src, real* const u[3], const adj* oa, adj* sa, adj* ua[3]) {
    SB s = to_sb(sb); VB v = to_vb(&c->velocity_boundary); advect_scalar_vjp(c, to_grid(&c->grid), &s, &v, src, u, oa, sa, ua);
}
EXPORT void og_advect_velocity_jvp(const og_config* c, real* const u[3], real* const ut[3], real* out[3]) { VB b = to_vb(&c->velocity_boundary); advect_velocity_jvp(c, to_grid(&c->grid), &b, u, ut, out); }
EXPORT void og_advect_scalar_jvp(const og_config* c, const og_sbnd* sb, const real* src, const real* srct, real* const u[3], real* const ut[3], real* out) {
    SB s = to_sb(sb); VB v = to_vb(&c->velocity_boundary); advect_scalar_jvp(c, to_grid(&c->grid), &s, &v, src, srct, u, ut, out);
}
EXPORT void og_projection_vjp(const og_config* c, adj* const oa[3], adj* pa, adj* ra, adj* ua[3], og_solve_stats* st) {
    SB b = to_sb(&c->pressure_boundary); projection_vjp(c, to_grid(&c->grid), &b, oa, pa, ra, ua, st);
}

/* ------------------------------------------------------------------------ */
/* domain build (model.cpp:32-155)                                           */
/* ------------------------------------------------------------------------ */
typedef struct {
    uint32_t shape;       /* 0 ellipsoid (data.ixx:55-58), 1 box (:60-63) */
    double center[3];
    double size[3];       /* radius or half extent */
    double velocity[3];
    double density, temperature;
} og_collider;

/* model.cpp:17-26, 49-77, 79-155.  Outputs: mask (N), collider face velocity
 * (3 face arrays), collider density/temperature (N); returns the anchor. */
EXPORT uint32_t og_build_domain(const og_grid* gg, const og_sbnd* pressure_boundary, const og_collider* colliders, uint32_t count,
                                uint32_t* mask, real* fv[3], real* cd, real* ct) {
    G g = to_grid(gg);
    size_t n = cells(g);
    real* cv = calloc(3 * n, sizeof(real));
    for (size_t i = 0; i < n; ++i) { mask[i] = 0; cd[i] = 0; ct[i] = 0; }
    for (int z = 0; z < g.nz; ++z) for (int y = 0; y < g.ny; ++y) for (int x = 0; x < g.nx; ++x) {
        size_t i = idx3(x, y, z, g.nx, g.ny);
        float px = ((float)x + 0.5F) * (float)gg->cell_size, py = ((float)y + 0.5F) * (float)gg->cell_size, pz = ((float)z + 0.5F) * (float)gg->cell_size;
        for (uint32_t k = 0; k < count; ++k) {
            const og_collider* cl = &colliders[k];
            int inside;
            if (cl->shape == 0) {
                float a = (px - (float)cl->center[0]) / (float)cl->size[0], b = (py - (float)cl->center[1]) / (float)cl->size[1], c = (pz - (float)cl->center[2]) / (float)cl->size[2];
                inside = a * a + b * b + c * c <= 1.0F;
            } else {
                inside = fabsf(px - (float)cl->center[0]) <= (float)cl->size[0] && fabsf(py - (float)cl->center[1]) <= (float)cl->size[1] && fabsf(pz - (float)cl->center[2]) <= (float)cl->size[2];
            }
            if (!inside) continue;
            mask[i] = 1u;
            cv[3 * i] = (real)cl->velocity[0]; cv[3 * i + 1] = (real)cl->velocity[1]; cv[3 * i + 2] = (real)cl->velocity[2];
            cd[i] = (real)cl->density; ct[i] = (real)cl->temperature;
        }
    }
    int fixed = 0;
    for (int f = 0; f < 6; ++f) if (pressure_boundary->modes[f] == 0u) fixed = 1;
    uint32_t anchor = 0;
    if (fixed) anchor = (uint32_t)n;
    else while (anchor < n && mask[anchor] != 0u) ++anchor;
    for (int a = 0; a < 3; ++a) {
        int ex = extent(g, a, 0), ey = extent(g, a, 1), ez = extent(g, a, 2);
        for (int z = 0; z < ez; ++z) for (int y = 0; y < ey; ++y) for (int x = 0; x < ex; ++x) {
            real sum = 0, cnt = 0;
            int c0[3] = {x - (a == 0), y - (a == 1), z - (a == 2)};
            if (in_grid(g, c0[0], c0[1], c0[2])) { size_t c = idx3(c0[0], c0[1], c0[2], g.nx, g.ny); if (mask[c]) { sum += cv[3 * c + a]; cnt += 1; } }
            if (in_grid(g, x, y, z)) { size_t c = idx3(x, y, z, g.nx, g.ny); if (mask[c]) { sum += cv[3 * c + a]; cnt += 1; } }
            fv[a][idx3(x, y, z, ex, ey)] = cnt == 0 ? (real)0 : sum / cnt;
        }
    }
    free(cv);
    return anchor;
}

/* ------------------------------------------------------------------------ */
/* step composition (model.cpp:341-389)                                      */
/* ------------------------------------------------------------------------ */
typedef struct {
    real* raw_advected[3];
    real* pressure;
    real* rhs;
} og_scratch;

/* model.cpp:341-349 */
EXPORT void og_forward_step(const og_config* c, const og_state* s, const og_control* u, const og_params* pr, og_state* next, og_cache* k,
                            og_scratch* w, og_solve_stats* st) {
    G g = to_grid(&c->grid);
    VB vb = to_vb(&c->velocity_boundary);
    SB pb = to_sb(&c->pressure_boundary), db = to_sb(&c->density_boundary), tb = to_sb(&c->temperature_boundary);
    source_forward(c, g, s->density, u->density_source, k->sourced_density, 0);
    source_forward(c, g, s->temperature, u->temperature_source, k->sourced_temperature, 1);
    buoyancy_forward(c, g, k->sourced_density, k->sourced_temperature, u->acceleration, pr, k->force);
    if (c->vorticity_enabled) vorticity_forward(c, g, s->velocity, pr->vorticity_confinement, k, k->force);
    integrate(c, g, s->velocity, k->force, k->forced_velocity);
    advect_velocity(c, g, &vb, k->forced_velocity, w->raw_advected);
    constrain(c, g, &vb, (real* const*)c->collider_velocity, w->raw_advected, k->advected_velocity);
    projection_forward(c, g, &pb, k->advected_velocity, w->pressure, w->rhs, next->velocity, st);
    advect_scalar(c, g, &db, &vb, c->collider_density, k->sourced_density, next->velocity, next->density);
    advect_scalar(c, g, &tb, &vb, c->collider_temperature, k->sourced_temperature, next->velocity, next->temperature);
}

/* model.cpp:351-359; scratch: 2N (sourced tangents) + 3N (force) + 3F*3
 * (forced, raw, advected tangents) + 2N (pressure, rhs) + 10N (vorticity) */
EXPORT void og_jvp_step(const og_config* c, const og_state* s, const og_params* pr, const og_state* next, const og_cache* k,
                        const og_state_tan* st, const og_control_tan* ct, const og_params* pt, og_state_tan* nt, real* scratch) {
    G g = to_grid(&c->grid);
    VB vb = to_vb(&c->velocity_boundary);
    SB pb = to_sb(&c->pressure_boundary), db = to_sb(&c->density_boundary), tb = to_sb(&c->temperature_boundary);
    SB pbt = zero_values_s(&pb);
    size_t n = cells(g), f0 = faces(g, 0), f1 = faces(g, 1), f2 = faces(g, 2);
    real* q = scratch;
    real* srt = q; q += n;
    real* sTt = q; q += n;
    real* ft[3] = {q, q + n, q + 2 * n}; q += 3 * n;
    real* fvt[3] = {q, q + f0, q + f0 + f1}; q += f0 + f1 + f2;
    real* rat[3] = {q, q + f0, q + f0 + f1}; q += f0 + f1 + f2;
    real* avt[3] = {q, q + f0, q + f0 + f1}; q += f0 + f1 + f2;
    real* ptn = q; q += n;
    real* rhst = q; q += n;
    real* vsc = q;
    source_jvp(c, g, st->density, ct->density_source, srt);
    source_jvp(c, g, st->temperature, ct->temperature_source, sTt);
    buoyancy_jvp(c, g, k->sourced_density, k->sourced_temperature, srt, sTt, ct->acceleration, pr, pt, ft);
    if (c->vorticity_enabled) vorticity_jvp(c, g, st->velocity, pr->vorticity_confinement, pt->vorticity_confinement, k, ft, vsc);
    integrate(c, g, st->velocity, ft, fvt);
    advect_velocity_jvp(c, g, &vb, k->forced_velocity, fvt, rat);
    VB vbt = zero_values_v(&vb);
    constrain(c, g, &vbt, NULL, rat, avt);
    projection_forward(c, g, &pbt, avt, ptn, rhst, nt->velocity, NULL);
    advect_scalar_jvp(c, g, &db, &vb, k->sourced_density, srt, next->velocity, nt->velocity, nt->density);
    advect_scalar_jvp(c, g, &tb, &vb, k->sourced_temperature, sTt, next->velocity, nt->velocity, nt->temperature);
}

/* model.cpp:361-389.  prev/ctrl/par are accumulated into (callers zero them
 * as solver.ixx:119-124, 143 do).  scratch: 2N + 3N + 4*3F + 2N + 10N adjoints. */
EXPORT void og_vjp_step(const og_config* c, const og_state* s, const og_params* pr, const og_state* next, const og_cache* k,
                        const og_state_adj* na, og_state_adj* prev, og_control_adj* ca, og_params_adj* pa, adj* scratch, og_solve_stats* stats) {
    G g = to_grid(&c->grid);
    VB vb = to_vb(&c->velocity_boundary);
    SB pb = to_sb(&c->pressure_boundary), db = to_sb(&c->density_boundary), tb = to_sb(&c->temperature_boundary);
    size_t n = cells(g), f0 = faces(g, 0), f1 = faces(g, 1), f2 = faces(g, 2), F = f0 + f1 + f2;
    memset(scratch, 0, (2 * n + 3 * n + 4 * F + 2 * n + 10 * n) * sizeof(adj));
    adj* q = scratch;
    adj* sra = q; q += n;
    adj* sTa = q; q += n;
    adj* fa[3] = {q, q + n, q + 2 * n}; q += 3 * n;
    adj* pva[3] = {q, q + f0, q + f0 + f1}; q += F;
    adj* ava[3] = {q, q + f0, q + f0 + f1}; q += F;
    adj* rva[3] = {q, q + f0, q + f0 + f1}; q += F;
    adj* fva[3] = {q, q + f0, q + f0 + f1}; q += F;
    adj* pra = q; q += n;
    adj* rha = q; q += n;
    adj* vsc = q;
    memcpy(pva[0], na->velocity[0], f0 * sizeof(adj));
    memcpy(pva[1], na->velocity[1], f1 * sizeof(adj));
    memcpy(pva[2], na->velocity[2], f2 * sizeof(adj));
    advect_scalar_vjp(c, g, &db, &vb, k->sourced_density, next->velocity, na->density, sra, pva);
    advect_scalar_vjp(c, g, &tb, &vb, k->sourced_temperature, next->velocity, na->temperature, sTa, pva);
    projection_vjp(c, g, &pb, pva, pra, rha, ava, stats);
    constrain_vjp(c, g, &vb, ava, rva);
    advect_velocity_vjp(c, g, &vb, k->forced_velocity, rva, fva);
    integrate_vjp(c, g, fva, prev->velocity, fa);
    buoyancy_vjp(c, g, k->sourced_density, k->sourced_temperature, pr, fa, sra, sTa, ca->acceleration, pa);
    if (c->vorticity_enabled) vorticity_vjp(c, g, pr->vorticity_confinement, k, fa, prev->velocity, &pa->vorticity_confinement, vsc);
    source_vjp(c, g, sra, prev->density, ca->density_source);
    source_vjp(c, g, sTa, prev->temperature, ca->temperature_source);
}

EXPORT int og_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n; return 1;
#endif
}
EXPORT size_t og_sizeof_config(void) { return sizeof(og_config); }
EXPORT size_t og_sizeof_real(void) { return sizeof(real); }
