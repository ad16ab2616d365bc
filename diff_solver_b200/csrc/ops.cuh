// Launchers shared between the kernel translation units and the step
// composition.  All enqueue on `st` and return an XsStatus.
#pragma once

#include "common.cuh"
#include "pressure.cuh"

namespace xs {

InflowSet make_inflows(const XsInflow* inflows, uint32_t count);

// forward.cu
XsStatus launch_source_buoyancy(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho, const float* temp,
                                const float* rho_src, const float* temp_src, const XsVector& acc, const float* ambient,
                                const float* beta_rho, const float* beta_temp, const InflowSet& inflows, float* rho_out,
                                float* temp_out, const XsVector& force);
XsStatus launch_integrate(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const XsVector& f, const XsVector& out);
XsStatus launch_advect_constrain(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& col, const XsVector& u,
                                 const XsVelocityBoundary& b, const XsVector& out);
XsStatus launch_advect_scalar_pair(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* col_rho, const float* col_temp,
                                   const float* src_rho, const float* src_temp, const XsVector& u, const XsScalarBoundary& rb,
                                   const XsScalarBoundary& tb, const XsVelocityBoundary& vb, float* out_rho, float* out_temp);
XsStatus launch_pressure_rhs(cudaStream_t st, const Grid& g, uint32_t anchor, const uint32_t* mask, const XsVector& u, float* rhs);
XsStatus launch_project(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const float* p, const XsVector& out);
XsStatus launch_project64(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const double* p, const XsVector& out);

// vorticity.cu
XsStatus vorticity_forward(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const float* conf, float* cache,
                           const XsVector& force);
XsStatus vorticity_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& ut, const float* conf, const float* conf_t,
                       const float* cache, const XsVector& force_t, float* scratch);
XsStatus vorticity_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* conf, const float* cache, const XsAdjointVector& fa,
                       const XsAdjointVector& ua, double* conf_adj, double* scratch);

// adjoint.cu
XsStatus launch_source_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const double* oa, const InflowSet& inflows, double* sa,
                           double* ra);
XsStatus launch_buoyancy_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho, const float* temp, const float* ambient,
                             const float* beta_rho, const float* beta_temp, const XsAdjointVector& fa, double* rho_a, double* temp_a,
                             const XsAdjointVector& ea, double* amb_a, double* br_a, double* bt_a);
// assign_force / assign: the force / velocity adjoint is written instead of
// accumulated (the step's scratch adjoints, which start at zero)
XsStatus launch_integrate_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsAdjointVector& oa, const XsAdjointVector& ua,
                              const XsAdjointVector& fa, bool assign_force = false);
XsStatus launch_advect_velocity_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const XsVelocityBoundary& vb,
                                    const XsAdjointVector& oa, const XsAdjointVector& ua);
XsStatus launch_advect_scalar_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* src, const XsScalarBoundary& sb,
                                  const double* oa, double* sa, const float* src2, const XsScalarBoundary& sb2, const double* oa2,
                                  double* sa2, const XsVector& u, const XsVelocityBoundary& vb, const XsAdjointVector& ua);
XsStatus launch_constrain_vjp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsAdjointVector& oa, const XsVelocityBoundary& b,
                              const XsAdjointVector& ua, bool assign = false);
XsStatus projection_vjp(cudaStream_t st, const Grid& g, const XsPressureSolve& solve, uint32_t anchor, const uint32_t* mask,
                        const XsAdjointVector& oa, const XsScalarBoundary& pb, double* pa, double* ra, const XsAdjointVector& ua,
                        void* workspace, const WarmHistory* history = nullptr, bool assign = false);

// tangent.cu
XsStatus launch_source_jvp_pair(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho_t, const float* temp_t,
                                const float* rho_src_t, const float* temp_src_t, const InflowSet& inflows, float* rho_out,
                                float* temp_out);
XsStatus launch_buoyancy_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* rho, const float* temp, const float* rho_t,
                             const float* temp_t, const XsVector& acc_t, const float* ambient, const float* beta_rho,
                             const float* beta_temp, const float* ambient_t, const float* beta_rho_t, const float* beta_temp_t,
                             const XsVector& force_t);
XsStatus launch_advect_velocity_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& u, const XsVector& ut,
                                    const XsVelocityBoundary& vb, const XsVector& out);
XsStatus launch_constrain(cudaStream_t st, const Grid& g, const uint32_t* mask, const XsVector& col, const XsVector& u,
                          const XsVelocityBoundary& b, const XsVector& out);
XsStatus launch_advect_scalar_jvp(cudaStream_t st, const Grid& g, const uint32_t* mask, const float* src, const float* src_t,
                                  const XsScalarBoundary& sb, float* out, const float* src2, const float* src2_t,
                                  const XsScalarBoundary& sb2, float* out2, const XsVector& u, const XsVector& ut,
                                  const XsVelocityBoundary& vb);

// projection forward with any solver kind (step.cu)
XsStatus projection_forward(cudaStream_t st, const Grid& g, const XsPressureSolve& solve, uint32_t anchor, const uint32_t* mask,
                            const XsVector& u, const XsScalarBoundary& pb, float* pressure, float* rhs, const XsVector& out,
                            void* workspace, cudaEvent_t begin = nullptr, cudaEvent_t end = nullptr, struct WarmStartNet* warm_start = nullptr,
                            const WarmHistory* history = nullptr, cudaEvent_t* stages = nullptr);

// Records stage event k of an optional event array (xs_smoke_forward_step's
// stage_events).
inline XsStatus mark_stage(cudaStream_t st, cudaEvent_t* events, int k) {
    if (events == nullptr || events[k] == nullptr) return XS_OK;
    return cudaEventRecord(events[k], st) == cudaSuccess ? XS_OK : XS_CUDA_ERROR;
}

}  // namespace xs
