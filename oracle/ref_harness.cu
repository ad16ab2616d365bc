// Reference-kernel harness.  TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference's own kernel file (solvers/smoke/operators.cu of
// diff-solver, included from where it lies, unmodified) for sm_100a and
// restates the reference's step composition (solvers/smoke/model.cpp:
// 341-389) around its launchers, behind a small C ABI that the GPU parity
// tests and the golden-vector generator call through ctypes.  The
// reference's host modules (model.cpp, operators.cpp, cuda.cpp) use
// `import std` and cannot be built with this toolchain; this file replaces
// only their call order.  Built by oracle/build_ref.sh into oracle/_ref/.
#include "operators.cu"
// The forward example driver's kernels (examples/smoke/forward/simulation.cu:
// write_control, reduce_metrics), also included unmodified.
#include "simulation.cu"

#include <cmath>
#include <cstdint>
#include <cstring>
#include <exception>

using namespace xayah::smoke::cuda_kernels;

extern "C" {

struct RefModel {
    Grid grid;
    VelocityBoundaryData velocity_boundary;
    ScalarBoundaryData pressure_boundary;
    ScalarBoundaryData density_boundary;
    ScalarBoundaryData temperature_boundary;
    uint32_t vorticity_enabled;
    uint32_t pressure_anchor;
    uint32_t iterations;
    const uint32_t* cell_mask;
    float* collider_velocity[3];
    float* collider_density;
    float* collider_temperature;
};

struct RefState { float* density; float* temperature; float* velocity[3]; };
struct RefControl { float* density_source; float* temperature_source; float* acceleration[3]; };
struct RefParams { float* ambient; float* density_buoyancy; float* temperature_buoyancy; float* confinement; };
struct RefCache {
    float* sourced_density; float* sourced_temperature; float* force[3]; float* vorticity;
    float* forced_velocity[3]; float* advected_velocity[3];
};
struct RefStateAdj { double* density; double* temperature; double* velocity[3]; };
struct RefControlAdj { double* density_source; double* temperature_source; double* acceleration[3]; };
struct RefParamsAdj { double* ambient; double* density_buoyancy; double* temperature_buoyancy; double* confinement; };

}  // extern "C"

namespace harness {

uint64_t cells(const Grid& g) { return static_cast<uint64_t>(g.nx) * g.ny * g.nz; }
uint64_t faces(const Grid& g, int a) {
    return static_cast<uint64_t>(g.nx + (a == 0)) * (g.ny + (a == 1)) * (g.nz + (a == 2));
}

VorticityView vort_view(float* base, uint64_t n) {
    return {{base, base + n, base + 2 * n}, {base + 3 * n, base + 4 * n, base + 5 * n}, {base + 6 * n},
            {base + 7 * n, base + 8 * n, base + 9 * n}, {base + 10 * n}};
}
ConstVorticityView const_vort_view(float* base, uint64_t n) {
    return {{base, base + n, base + 2 * n}, {base + 3 * n, base + 4 * n, base + 5 * n}, {base + 6 * n},
            {base + 7 * n, base + 8 * n, base + 9 * n}, {base + 10 * n}};
}

// Scratch carving: forward needs raw advected (F), pressure and rhs (2N);
// the tangent pass 2N + 3N + 3F + 2N + 10N floats; the adjoint pass
// 2N + 3N + 4F + 2N + 10N doubles.
struct Carve {
    char* p;
    size_t off;
    template <class T>
    T* take(uint64_t count) {
        T* r = p ? reinterpret_cast<T*>(p + off) : nullptr;
        off += (count * sizeof(T) + 255) / 256 * 256;
        return r;
    }
};

// FP64 relative residual of the RBGS system for the FP32 pressure, one
// partial per block (harness-only helper).
__global__ void residual_kernel(const Grid grid, const uint32_t anchor, const uint32_t* mask, const ScalarBoundaryData boundary,
                                const float* rhs, const float* pressure, double* partial) {
    __shared__ double sb[256], sr[256];
    const uint64_t index = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double b2 = 0.0, r2 = 0.0;
    if (index < cell_count(grid) && (mask == nullptr || mask[index] == 0u) && index != anchor) {
        int x, y, z;
        decode(index, grid.nx, grid.ny, x, y, z);
        double sum = rhs[index], diag = 0.0, fixed = 0.0;
        for (int d = 0; d < 3; ++d)
            for (int dir = -1; dir <= 1; dir += 2) {
                int nx, ny, nz; bool connected, fx; float fv{};
                pressure_neighbor(grid, boundary, mask, x, y, z, d, dir, nx, ny, nz, connected, fx, fv);
                if (connected) { sum += pressure[index3(nx, ny, nz, grid.nx, grid.ny)]; diag += 1.0; }
                else if (fx) { fixed += fv; diag += 1.0; }
            }
        if (diag > 0.0) {
            const double b = static_cast<double>(rhs[index]) + fixed;
            const double r = sum + fixed - diag * pressure[index];
            b2 = b * b;
            r2 = r * r;
        }
    }
    sb[threadIdx.x] = b2;
    sr[threadIdx.x] = r2;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) { sb[threadIdx.x] += sb[threadIdx.x + s]; sr[threadIdx.x] += sr[threadIdx.x + s]; }
        __syncthreads();
    }
    if (threadIdx.x == 0) { partial[2 * blockIdx.x] = sb[0]; partial[2 * blockIdx.x + 1] = sr[0]; }
}

}  // namespace harness

using namespace harness;

extern "C" {

size_t ref_scratch_bytes(const RefModel* m) {
    const Grid& g = m->grid;
    const uint64_t n = cells(g), F = faces(g, 0) + faces(g, 1) + faces(g, 2);
    return 4 * (F + 2 * n) + 4 * (17 * n + 3 * F) + 8 * (17 * n + 4 * F) + 64 * 1024 + 8 * 2 * ((n + 255) / 256) + 4096;
}

// Relative residual of `pressure` for `rhs` (FP64, harness kernel).
double ref_relative_residual(cudaStream_t stream, const RefModel* m, const float* rhs, const float* pressure, double* partial_scratch) {
    const Grid& g = m->grid;
    const unsigned nb = static_cast<unsigned>((cells(g) + 255) / 256);
    residual_kernel<<<nb, 256, 0, stream>>>(g, m->pressure_anchor, m->cell_mask, m->pressure_boundary, rhs, pressure, partial_scratch);
    double* host = new double[2 * nb];
    cudaMemcpyAsync(host, partial_scratch, sizeof(double) * 2 * nb, cudaMemcpyDeviceToHost, stream);
    cudaStreamSynchronize(stream);
    double b = 0.0, r = 0.0;
    for (unsigned i = 0; i < nb; ++i) { b += host[2 * i]; r += host[2 * i + 1]; }
    delete[] host;
    return b > 0.0 ? std::sqrt(r / b) : 0.0;
}

// projection_forward (operators.cu:1004-1013) with the RBGS loop run until
// the FP64 relative residual reaches `tolerance` (checked every `check`
// sweep pairs), or `max_sweeps` pairs, or until a check window no longer
// lowers the residual by 0.1 % (the FP32 iteration has reached its rounding
// floor).  Returns sweeps taken.
uint32_t ref_projection_converged(cudaStream_t stream, const RefModel* m, float* const u[3], float* pressure, float* rhs, float* out[3],
                                  double tolerance, uint32_t max_sweeps, uint32_t check, double* partial_scratch, double* residual_out) {
    const Grid& g = m->grid;
    const uint64_t n = cells(g);
    const unsigned nb = static_cast<unsigned>((n + 255) / 256);
    cudaMemsetAsync(pressure, 0, n * sizeof(float), stream);
    ConstStaggeredVectorView vel{u[0], u[1], u[2]};
    pressure_rhs_kernel<<<nb, 256, 0, stream>>>(g, m->pressure_anchor, m->cell_mask, vel, rhs);
    uint32_t sweeps = 0;
    double res = ref_relative_residual(stream, m, rhs, pressure, partial_scratch);
    while (res > tolerance && sweeps < max_sweeps) {
        for (uint32_t k = 0; k < check && sweeps < max_sweeps; ++k, ++sweeps) {
            rbgs_kernel<<<nb, 256, 0, stream>>>(g, 0, m->pressure_anchor, m->cell_mask, m->pressure_boundary, rhs, pressure);
            rbgs_kernel<<<nb, 256, 0, stream>>>(g, 1, m->pressure_anchor, m->cell_mask, m->pressure_boundary, rhs, pressure);
        }
        const double previous = res;
        res = ref_relative_residual(stream, m, rhs, pressure, partial_scratch);
        if (res > 0.999 * previous) break;
    }
    for (int a = 0; a < 3; ++a) {
        const unsigned fb = static_cast<unsigned>((faces(g, a) + 255) / 256);
        project_velocity_kernel<<<fb, 256, 0, stream>>>(g, a, m->cell_mask, u[a], pressure, out[a]);
    }
    if (residual_out) *residual_out = res;
    return sweeps;
}

// Model::forward_step (model.cpp:341-349).  tolerance > 0 runs RBGS to that
// relative residual instead of m->iterations sweeps.
int ref_forward_step(cudaStream_t stream, const RefModel* m, RefState s, RefControl c, RefParams p, RefState next, RefCache k,
                     void* scratch, double tolerance, uint32_t max_sweeps, uint32_t* sweeps_out, double* residual_out) {
    try {
        const Grid& g = m->grid;
        const uint64_t n = cells(g);
        Carve cv{static_cast<char*>(scratch), 0};
        float* raw[3] = {cv.take<float>(faces(g, 0)), cv.take<float>(faces(g, 1)), cv.take<float>(faces(g, 2))};
        float* pressure = cv.take<float>(n);
        float* rhs = cv.take<float>(n);
        double* partial = cv.take<double>(2 * ((n + 255) / 256));
        const uint32_t* mask = m->cell_mask;
        source_forward(stream, g, mask, {s.density}, {c.density_source}, {k.sourced_density});
        source_forward(stream, g, mask, {s.temperature}, {c.temperature_source}, {k.sourced_temperature});
        buoyancy_forward(stream, g, mask, {k.sourced_density}, {k.sourced_temperature},
                         {c.acceleration[0], c.acceleration[1], c.acceleration[2]}, p.ambient, p.density_buoyancy, p.temperature_buoyancy,
                         {k.force[0], k.force[1], k.force[2]});
        if (m->vorticity_enabled)
            vorticity_forward(stream, g, mask, {s.velocity[0], s.velocity[1], s.velocity[2]}, p.confinement, vort_view(k.vorticity, n),
                              {k.force[0], k.force[1], k.force[2]});
        integrate_velocity_forward(stream, g, mask, {s.velocity[0], s.velocity[1], s.velocity[2]}, {k.force[0], k.force[1], k.force[2]},
                                   {k.forced_velocity[0], k.forced_velocity[1], k.forced_velocity[2]});
        advect_velocity_forward(stream, g, mask, {k.forced_velocity[0], k.forced_velocity[1], k.forced_velocity[2]}, m->velocity_boundary,
                                {raw[0], raw[1], raw[2]});
        constrain_velocity_forward(stream, g, mask, {m->collider_velocity[0], m->collider_velocity[1], m->collider_velocity[2]},
                                   {raw[0], raw[1], raw[2]}, m->velocity_boundary,
                                   {k.advected_velocity[0], k.advected_velocity[1], k.advected_velocity[2]});
        if (tolerance > 0.0) {
            const uint32_t sw = ref_projection_converged(stream, m, k.advected_velocity, pressure, rhs, next.velocity, tolerance, max_sweeps, 50,
                                                         partial, residual_out);
            if (sweeps_out) *sweeps_out = sw;
        } else {
            projection_forward(stream, g, m->iterations, m->pressure_anchor, mask,
                               {k.advected_velocity[0], k.advected_velocity[1], k.advected_velocity[2]}, m->velocity_boundary,
                               m->pressure_boundary, {pressure}, {rhs}, {next.velocity[0], next.velocity[1], next.velocity[2]});
            if (sweeps_out) *sweeps_out = m->iterations;
            if (residual_out) *residual_out = ref_relative_residual(stream, m, rhs, pressure, partial);
        }
        advect_scalar_forward(stream, g, mask, {m->collider_density}, {k.sourced_density}, {next.velocity[0], next.velocity[1], next.velocity[2]},
                              m->density_boundary, m->velocity_boundary, {next.density});
        advect_scalar_forward(stream, g, mask, {m->collider_temperature}, {k.sourced_temperature},
                              {next.velocity[0], next.velocity[1], next.velocity[2]}, m->temperature_boundary, m->velocity_boundary,
                              {next.temperature});
    } catch (const std::exception&) {
        return 1;
    }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

// Model::jvp_step (model.cpp:351-359)
int ref_jvp_step(cudaStream_t stream, const RefModel* m, RefState s, RefParams p, RefState next, RefCache k, RefState st, RefControl ct,
                 RefParams pt, RefState nt, void* scratch) {
    (void)s;
    try {
        const Grid& g = m->grid;
        const uint64_t n = cells(g);
        Carve cv{static_cast<char*>(scratch), 0};
        cv.take<float>(faces(g, 0) + faces(g, 1) + faces(g, 2) + 2 * n);  // forward part
        float* srt = cv.take<float>(n);
        float* sTt = cv.take<float>(n);
        float* ft[3] = {cv.take<float>(n), cv.take<float>(n), cv.take<float>(n)};
        float* fvt[3] = {cv.take<float>(faces(g, 0)), cv.take<float>(faces(g, 1)), cv.take<float>(faces(g, 2))};
        float* rat[3] = {cv.take<float>(faces(g, 0)), cv.take<float>(faces(g, 1)), cv.take<float>(faces(g, 2))};
        float* avt[3] = {cv.take<float>(faces(g, 0)), cv.take<float>(faces(g, 1)), cv.take<float>(faces(g, 2))};
        float* ptn = cv.take<float>(n);
        float* rhst = cv.take<float>(n);
        float* vs = cv.take<float>(10 * n);
        const uint32_t* mask = m->cell_mask;
        source_jvp(stream, g, mask, {st.density}, {ct.density_source}, {srt});
        source_jvp(stream, g, mask, {st.temperature}, {ct.temperature_source}, {sTt});
        buoyancy_jvp(stream, g, mask, {k.sourced_density}, {k.sourced_temperature}, {srt}, {sTt},
                     {ct.acceleration[0], ct.acceleration[1], ct.acceleration[2]}, p.ambient, p.density_buoyancy, p.temperature_buoyancy,
                     pt.ambient, pt.density_buoyancy, pt.temperature_buoyancy, {ft[0], ft[1], ft[2]});
        if (m->vorticity_enabled) {
            VorticityTangentScratch ts{{vs, vs + n, vs + 2 * n}, {vs + 3 * n, vs + 4 * n, vs + 5 * n}, {vs + 6 * n},
                                       {vs + 7 * n, vs + 8 * n, vs + 9 * n}};
            vorticity_jvp(stream, g, mask, {st.velocity[0], st.velocity[1], st.velocity[2]}, p.confinement, pt.confinement,
                          const_vort_view(k.vorticity, n), {ft[0], ft[1], ft[2]}, ts);
        }
        integrate_velocity_jvp(stream, g, mask, {st.velocity[0], st.velocity[1], st.velocity[2]}, {ft[0], ft[1], ft[2]}, {fvt[0], fvt[1], fvt[2]});
        advect_velocity_jvp(stream, g, mask, {k.forced_velocity[0], k.forced_velocity[1], k.forced_velocity[2]}, {fvt[0], fvt[1], fvt[2]},
                            m->velocity_boundary, {rat[0], rat[1], rat[2]});
        constrain_velocity_jvp(stream, g, mask, {rat[0], rat[1], rat[2]}, m->velocity_boundary, {avt[0], avt[1], avt[2]});
        projection_jvp(stream, g, m->iterations, m->pressure_anchor, mask, {avt[0], avt[1], avt[2]}, m->velocity_boundary, m->pressure_boundary,
                       {ptn}, {rhst}, {nt.velocity[0], nt.velocity[1], nt.velocity[2]});
        advect_scalar_jvp(stream, g, mask, {k.sourced_density}, {srt}, {next.velocity[0], next.velocity[1], next.velocity[2]},
                          {nt.velocity[0], nt.velocity[1], nt.velocity[2]}, m->density_boundary, m->velocity_boundary, {nt.density});
        advect_scalar_jvp(stream, g, mask, {k.sourced_temperature}, {sTt}, {next.velocity[0], next.velocity[1], next.velocity[2]},
                          {nt.velocity[0], nt.velocity[1], nt.velocity[2]}, m->temperature_boundary, m->velocity_boundary, {nt.temperature});
    } catch (const std::exception&) {
        return 1;
    }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

// Model::vjp_step (model.cpp:361-389); accumulates into pa, ca, qa.
int ref_vjp_step(cudaStream_t stream, const RefModel* m, RefState s, RefParams p, RefState next, RefCache k, RefStateAdj na,
                 RefStateAdj pa, RefControlAdj ca, RefParamsAdj qa, void* scratch) {
    try {
        const Grid& g = m->grid;
        const uint64_t n = cells(g);
        const uint64_t f[3] = {faces(g, 0), faces(g, 1), faces(g, 2)};
        Carve cv{static_cast<char*>(scratch), 0};
        cv.take<float>(f[0] + f[1] + f[2] + 2 * n);
        cv.take<float>(17 * n + 3 * (f[0] + f[1] + f[2]));
        double* sra = cv.take<double>(n);
        double* sTa = cv.take<double>(n);
        double* fa[3] = {cv.take<double>(n), cv.take<double>(n), cv.take<double>(n)};
        double* pva[3] = {cv.take<double>(f[0]), cv.take<double>(f[1]), cv.take<double>(f[2])};
        double* ava[3] = {cv.take<double>(f[0]), cv.take<double>(f[1]), cv.take<double>(f[2])};
        double* rva[3] = {cv.take<double>(f[0]), cv.take<double>(f[1]), cv.take<double>(f[2])};
        double* fva[3] = {cv.take<double>(f[0]), cv.take<double>(f[1]), cv.take<double>(f[2])};
        double* pra = cv.take<double>(n);
        double* rha = cv.take<double>(n);
        double* vs = cv.take<double>(10 * n);
        const uint32_t* mask = m->cell_mask;
        cudaMemsetAsync(sra, 0, 8 * n, stream);
        cudaMemsetAsync(sTa, 0, 8 * n, stream);
        for (int a = 0; a < 3; ++a) {
            cudaMemsetAsync(fa[a], 0, 8 * n, stream);
            cudaMemsetAsync(ava[a], 0, 8 * f[a], stream);
            cudaMemsetAsync(rva[a], 0, 8 * f[a], stream);
            cudaMemsetAsync(fva[a], 0, 8 * f[a], stream);
            cudaMemcpyAsync(pva[a], na.velocity[a], 8 * f[a], cudaMemcpyDeviceToDevice, stream);
        }
        const ConstStaggeredVectorView nv{next.velocity[0], next.velocity[1], next.velocity[2]};
        advect_scalar_vjp(stream, g, mask, {k.sourced_density}, nv, m->density_boundary, m->velocity_boundary, {na.density}, {sra},
                          {pva[0], pva[1], pva[2]});
        advect_scalar_vjp(stream, g, mask, {k.sourced_temperature}, nv, m->temperature_boundary, m->velocity_boundary, {na.temperature}, {sTa},
                          {pva[0], pva[1], pva[2]});
        projection_vjp(stream, g, m->iterations, m->pressure_anchor, mask, {pva[0], pva[1], pva[2]}, m->velocity_boundary, m->pressure_boundary,
                       {pra}, {rha}, {ava[0], ava[1], ava[2]});
        constrain_velocity_vjp(stream, g, mask, {ava[0], ava[1], ava[2]}, m->velocity_boundary, {rva[0], rva[1], rva[2]});
        advect_velocity_vjp(stream, g, mask, {k.forced_velocity[0], k.forced_velocity[1], k.forced_velocity[2]}, m->velocity_boundary,
                            {rva[0], rva[1], rva[2]}, {fva[0], fva[1], fva[2]});
        integrate_velocity_vjp(stream, g, mask, {fva[0], fva[1], fva[2]}, {pa.velocity[0], pa.velocity[1], pa.velocity[2]}, {fa[0], fa[1], fa[2]});
        buoyancy_vjp(stream, g, mask, {k.sourced_density}, {k.sourced_temperature}, p.ambient, p.density_buoyancy, p.temperature_buoyancy,
                     {fa[0], fa[1], fa[2]}, {sra}, {sTa}, {ca.acceleration[0], ca.acceleration[1], ca.acceleration[2]}, qa.ambient,
                     qa.density_buoyancy, qa.temperature_buoyancy);
        if (m->vorticity_enabled) {
            VorticityAdjointScratch as{{vs, vs + n, vs + 2 * n}, {vs + 3 * n, vs + 4 * n, vs + 5 * n}, {vs + 6 * n},
                                       {vs + 7 * n, vs + 8 * n, vs + 9 * n}};
            vorticity_vjp(stream, g, mask, p.confinement, const_vort_view(k.vorticity, n), {fa[0], fa[1], fa[2]},
                          {pa.velocity[0], pa.velocity[1], pa.velocity[2]}, qa.confinement, as);
        }
        source_vjp(stream, g, mask, {sra}, {pa.density}, {ca.density_source});
        source_vjp(stream, g, mask, {sTa}, {pa.temperature}, {ca.temperature_source});
        (void)s;
    } catch (const std::exception&) {
        return 1;
    }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

// Single reference operators, for per-operator parity.
int ref_advect_velocity(cudaStream_t stream, const RefModel* m, float* const u[3], float* out[3]) {
    try {
        advect_velocity_forward(stream, m->grid, m->cell_mask, {u[0], u[1], u[2]}, m->velocity_boundary, {out[0], out[1], out[2]});
    } catch (const std::exception&) { return 1; }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

int ref_advect_scalar(cudaStream_t stream, const RefModel* m, const ScalarBoundaryData* sb, const float* col, const float* src,
                      float* const u[3], float* out) {
    try {
        advect_scalar_forward(stream, m->grid, m->cell_mask, {col}, {src}, {u[0], u[1], u[2]}, *sb, m->velocity_boundary, {out});
    } catch (const std::exception&) { return 1; }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

int ref_rbgs(cudaStream_t stream, const RefModel* m, const float* rhs, float* pressure, uint32_t sweeps) {
    const uint64_t n = cells(m->grid);
    const unsigned nb = static_cast<unsigned>((n + 255) / 256);
    for (uint32_t i = 0; i < sweeps; ++i) {
        rbgs_kernel<<<nb, 256, 0, stream>>>(m->grid, 0, m->pressure_anchor, m->cell_mask, m->pressure_boundary, rhs, pressure);
        rbgs_kernel<<<nb, 256, 0, stream>>>(m->grid, 1, m->pressure_anchor, m->cell_mask, m->pressure_boundary, rhs, pressure);
    }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

// The reference's vorticity_forward (operators.cu:973-979) alone.
int ref_vorticity_forward(cudaStream_t stream, const RefModel* m, float* const u[3], const float* confinement, float* cache, float* force[3]) {
    try {
        vorticity_forward(stream, m->grid, m->cell_mask, {u[0], u[1], u[2]}, confinement, vort_view(cache, cells(m->grid)),
                          {force[0], force[1], force[2]});
    } catch (const std::exception&) { return 1; }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

// One reference launcher, enqueued without synchronisation, for per-kernel
// timing with events on the stream.  `which`:
//   0 advect_velocity_forward (u -> out)      1 constrain_velocity_forward (u -> out)
//   2 advect_scalar_forward (src, u -> sout)  3 pressure_rhs (u -> rhs)
//   4 one red-black sweep pair (rhs, p)       5 project_velocity, 3 axes (u, p -> out)
//   6 advect_velocity_vjp (u, oa -> ua)       7 advect_scalar_vjp (src, u, soa -> sa, ua)
struct RefLaunchArgs {
    float* u[3];
    float* out[3];
    const float* src;
    float* sout;
    float* rhs;
    float* pressure;
    double* oa[3];
    double* ua[3];
    const double* soa;
    double* sa;
};

int ref_launch(cudaStream_t stream, const RefModel* m, uint32_t which, const RefLaunchArgs* a) {
    try {
        const Grid& g = m->grid;
        const uint32_t* mask = m->cell_mask;
        const unsigned nb = static_cast<unsigned>((cells(g) + 255) / 256);
        switch (which) {
            case 0:
                advect_velocity_forward(stream, g, mask, {a->u[0], a->u[1], a->u[2]}, m->velocity_boundary, {a->out[0], a->out[1], a->out[2]});
                break;
            case 1:
                constrain_velocity_forward(stream, g, mask, {m->collider_velocity[0], m->collider_velocity[1], m->collider_velocity[2]},
                                           {a->u[0], a->u[1], a->u[2]}, m->velocity_boundary, {a->out[0], a->out[1], a->out[2]});
                break;
            case 2:
                advect_scalar_forward(stream, g, mask, {m->collider_density}, {a->src}, {a->u[0], a->u[1], a->u[2]}, m->density_boundary,
                                      m->velocity_boundary, {a->sout});
                break;
            case 3:
                pressure_rhs_kernel<<<nb, 256, 0, stream>>>(g, m->pressure_anchor, mask, ConstStaggeredVectorView{a->u[0], a->u[1], a->u[2]},
                                                            a->rhs);
                break;
            case 4:
                rbgs_kernel<<<nb, 256, 0, stream>>>(g, 0, m->pressure_anchor, mask, m->pressure_boundary, a->rhs, a->pressure);
                rbgs_kernel<<<nb, 256, 0, stream>>>(g, 1, m->pressure_anchor, mask, m->pressure_boundary, a->rhs, a->pressure);
                break;
            case 5:
                for (int axis = 0; axis < 3; ++axis) {
                    const unsigned fb = static_cast<unsigned>((faces(g, axis) + 255) / 256);
                    project_velocity_kernel<<<fb, 256, 0, stream>>>(g, axis, mask, a->u[axis], a->pressure, a->out[axis]);
                }
                break;
            case 6:
                advect_velocity_vjp(stream, g, mask, {a->u[0], a->u[1], a->u[2]}, m->velocity_boundary, {a->oa[0], a->oa[1], a->oa[2]},
                                    {a->ua[0], a->ua[1], a->ua[2]});
                break;
            case 7:
                advect_scalar_vjp(stream, g, mask, {a->src}, {a->u[0], a->u[1], a->u[2]}, m->density_boundary, m->velocity_boundary, {a->soa},
                                  {a->sa}, {a->ua[0], a->ua[1], a->ua[2]});
                break;
            default:
                return 3;
        }
    } catch (const std::exception&) {
        return 1;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

// The example driver's launchers (simulation.cu:88-100).
int ref_write_control(cudaStream_t stream, const RefModel* m, uint64_t step, float pulse_period, const float* left_center,
                      const float* right_center, float source_radius, float density_rate, float temperature_rate, const float* left_acc,
                      const float* right_acc, float* density_source, float* temperature_source, float* acceleration[3]) {
    namespace ex = xayah::smoke::examples::forward::simulation_cuda;
    try {
        ex::launch_write_control(stream, m->grid, step, pulse_period, Vector{left_center[0], left_center[1], left_center[2]},
                                 Vector{right_center[0], right_center[1], right_center[2]}, source_radius, density_rate, temperature_rate,
                                 Vector{left_acc[0], left_acc[1], left_acc[2]}, Vector{right_acc[0], right_acc[1], right_acc[2]}, density_source,
                                 temperature_source, CenteredVectorView{acceleration[0], acceleration[1], acceleration[2]});
    } catch (const std::exception&) { return 1; }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

// reduce_metrics into metrics[6], zeroed first as simulation.cpp:97 does.
int ref_reduce_metrics(cudaStream_t stream, const RefModel* m, const float* density, const float* temperature, float* const pre[3],
                       float* const post[3], double* metrics) {
    namespace ex = xayah::smoke::examples::forward::simulation_cuda;
    try {
        cudaMemsetAsync(metrics, 0, 6 * sizeof(double), stream);
        ex::launch_reduce_metrics(stream, m->grid, m->cell_mask, density, temperature, ConstStaggeredVectorView{pre[0], pre[1], pre[2]},
                                  ConstStaggeredVectorView{post[0], post[1], post[2]}, metrics);
    } catch (const std::exception&) { return 1; }
    return cudaStreamSynchronize(stream) == cudaSuccess ? 0 : 2;
}

// Layout check: the harness' view of the model block as 32-bit words.
size_t ref_model_words(const RefModel* m, uint32_t* out, size_t capacity) {
    const size_t words = sizeof(RefModel) / 4;
    std::memcpy(out, m, 4 * (words < capacity ? words : capacity));
    return sizeof(RefModel);
}

}  // extern "C"
