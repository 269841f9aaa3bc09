// Tet-quality regularizer gradient (the reference's TetRegularizerPass:
// Data/Shaders/Optimizer/TetRegularizer.glsl:108-166, dispatched by
// TetRegularizerPass.cpp:94 and bound as difftetvr.TetRegularizer,
// Module.cpp:663-695 / 983-995).
//
// Per tet with vertices p0..p3 (cell order):
//   D = det[p1 - p0, p2 - p0, p3 - p0]       (6 V = -D in the reference's sign)
//   S = sum of the six squared edge lengths   (l_rms^2 = S / 6)
//   q = 6 sqrt(2) V / l_rms^3 = -c D / S^(3/2),  c = 12 sqrt(3)   (Parthasarathy et al. 1991)
//   L = (lambda / beta) log(1 + exp(-beta q))    (mirrored softplus: low quality is penalised)
//   dL/dq = -lambda / (1 + exp(beta q))
//   dq/dp = (-c S dD/dp + 1.5 c D dS/dp) / max(S^(5/2), 1e-5)
// with dD/dp1 = (p2 - p0) x (p3 - p0), dD/dp2 = (p3 - p0) x (p1 - p0),
// dD/dp3 = (p1 - p0) x (p2 - p0), dD/dp0 = -(their sum), and
// dS/dpi = 2 (4 pi - sum_j pj).  The denominator clamp is the reference's
// (TetRegularizer.glsl:140-142); it is active for tets with S < 0.01.
// The gradient is added into the position gradient [3V]; the loss (a value
// the reference does not compute) is optionally accumulated.
#include "dtv_host.h"
#include "dtv_internal.h"
#include "difftetvr_b200.h"

namespace dtv {

constexpr float kRegC = 20.784609690826528f;  // 12 sqrt(3)

__device__ __forceinline__ float3 sub3(float3 a, float3 b) { return make_float3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 cross3(float3 a, float3 b) {
    return make_float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float dot3(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

__global__ void __launch_bounds__(256) k_tet_regularizer(const uint4* __restrict__ cells, uint32_t T,
                                                         const float* __restrict__ pos, float lambda, float beta,
                                                         float* __restrict__ grad, float* __restrict__ loss) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    float l = 0.f;
    if (t < T) {
        const uint4 c = cells[t];
        const uint32_t vi[4] = {c.x, c.y, c.z, c.w};
        float3 p[4];
#pragma unroll
        for (int j = 0; j < 4; ++j)
            p[j] = make_float3(pos[3 * size_t(vi[j])], pos[3 * size_t(vi[j]) + 1], pos[3 * size_t(vi[j]) + 2]);
        const float3 e1 = sub3(p[1], p[0]), e2 = sub3(p[2], p[0]), e3 = sub3(p[3], p[0]);
        float3 dD[4];
        dD[1] = cross3(e2, e3);
        dD[2] = cross3(e3, e1);
        dD[3] = cross3(e1, e2);
        dD[0] = make_float3(-(dD[1].x + dD[2].x + dD[3].x), -(dD[1].y + dD[2].y + dD[3].y),
                            -(dD[1].z + dD[2].z + dD[3].z));
        const float D = dot3(dD[3], e3);
        const float3 e12 = sub3(p[2], p[1]), e13 = sub3(p[3], p[1]), e23 = sub3(p[3], p[2]);
        const float S = dot3(e1, e1) + dot3(e2, e2) + dot3(e3, e3) + dot3(e12, e12) + dot3(e13, e13) + dot3(e23, e23);
        const float s15 = S * sqrtf(S);
        const float q = -kRegC * D / s15;
        const float dLdq = -lambda / (1.f + expf(beta * q));
        const float den = fmaxf(S * s15, 1e-5f);
        const float a = -kRegC * S / den, b = 1.5f * kRegC * D / den;
        const float3 sum = make_float3(p[0].x + p[1].x + p[2].x + p[3].x, p[0].y + p[1].y + p[2].y + p[3].y,
                                       p[0].z + p[1].z + p[2].z + p[3].z);
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const float3 dS = make_float3(2.f * (4.f * p[j].x - sum.x), 2.f * (4.f * p[j].y - sum.y),
                                          2.f * (4.f * p[j].z - sum.z));
            float* g = grad + 3 * size_t(vi[j]);
            atomicAdd(g, dLdq * (a * dD[j].x + b * dS.x));
            atomicAdd(g + 1, dLdq * (a * dD[j].y + b * dS.y));
            atomicAdd(g + 2, dLdq * (a * dD[j].z + b * dS.z));
        }
        if (loss) {
            // (lambda / beta) softplus(-beta q), overflow-safe.
            const float z = -beta * q;
            l = (lambda / beta) * (fmaxf(z, 0.f) + log1pf(expf(-fabsf(z))));
        }
    }
    if (loss) {
        for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
        if ((threadIdx.x & 31) == 0 && l != 0.f) atomicAdd(loss, l);
    }
}

}  // namespace dtv

extern "C" int32_t dtv_tet_regularizer_grad(const dtv_mesh* mesh, const float* d_positions, float lambda,
                                            float beta, float* d_grad_positions, float* d_loss, dtv_stream stream) {
    using namespace dtv_host;
    return guarded([&] {
        require(mesh != nullptr, "mesh is null");
        require(d_positions && d_grad_positions, "null device pointer");
        require(beta > 0.f, "softplus beta must be > 0");
        const uint64_t T = dtv::mesh_num_cells(mesh);
        if (T == 0) return;
        dtv::k_tet_regularizer<<<unsigned((T + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
            reinterpret_cast<const uint4*>(dtv::mesh_cells_device(mesh)), uint32_t(T), d_positions, lambda, beta,
            d_grad_positions, d_loss);
        check_launch("tet regularizer");
    });
}
