// moist_bridge.cu - sm_100a kernel of the eqtset=2 moist stage terms:
// moist buoyancy, density potential temperature (theta-rho), the theta and
// pressure energy terms, and the advected Exner function piadv.
//
// Behaviour followed (reference file:line):
//   cpu_eqtset2_cell_f32           src/cm1core/cuda_moist_stage_bridge.py:62-139
//   array layouts of the stage-terms launch
//   launch_cuda_eqtset2_stage_terms src/cm1core/cuda_moist_stage_bridge.py:378-430
//
// Design (B200): one elementwise pass over the periodic-padded scalar box
// (nk levels x (nj+2) x (ni+2)); live cells produce all four terms, and every
// cell of the box (halos included) produces piadv from the nearest live
// base-state column, as the reference's piadv kernel does.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int kBX = 32, kBY = 4;

__global__ void __launch_bounds__(kBX *kBY)
    eqtset2_terms_kernel(gm1b_eqtset2_arrays a, int ni, int nj, int nk, int base3d) {
    const int x = blockIdx.x * kBX + threadIdx.x;  // 0..ni+1
    const int y = blockIdx.y * kBY + threadIdx.y;  // 0..nj+1
    const int k = blockIdx.z;                      // 0..nk-1 (level k+1 of padded arrays)
    if (x >= ni + 2 || y >= nj + 2) return;
    const size_t pp = ((size_t)(k + 1) * (nj + 2) + y) * (size_t)(ni + 2) + x;  // periodic-padded index
    const int ii = x < 1 ? 0 : (x > ni ? ni - 1 : x - 1);
    const int jj = y < 1 ? 0 : (y > nj ? nj - 1 : y - 1);
    const size_t cell = ((size_t)k * nj + jj) * (size_t)ni + ii;
    const size_t bidx = base3d ? cell : (size_t)k;
    const float bp = a.pi0[bidx];
    a.piadv[pp] = bp + a.pp3d[pp];
    if (x < 1 || x > ni || y < 1 || y > nj) return;
    const float rd = 287.04f, rv = 461.5f, cp = 1005.7f, cpv = 1870.0f, cpl = 4190.0f, cpi = 2106.0f, g = 9.81f;
    const float cv = cp - rd, cvv = cpv - rv, rovcp = rd / cp, reps = rv / rd;
    const float repsm1 = reps - 1.0f;
    const size_t n = (size_t)ni * nj * nk;
    const float qv = fmaxf(a.q3d[cell], 0.0f);
    const float liquid = a.q3d[n + cell] + a.q3d[2 * n + cell];
    const float ice = (a.q3d[3 * n + cell] + a.q3d[4 * n + cell]) + a.q3d[5 * n + cell];
    const float qli = fmaxf(liquid + ice, 0.0f);
    const float cpli = cpl * fmaxf(liquid, 0.0f) + cpi * fmaxf(ice, 0.0f);
    const float th0 = a.th0[bidx], qv0 = a.qv0[bidx];
    const float qc0 = a.qc0 ? a.qc0[bidx] : 0.0f, qi0 = a.qi0 ? a.qi0[bidx] : 0.0f;
    const float th3d = a.th3d[cell];
    const float theta = th0 + th3d;
    float b = th3d * (1.0f / th0) + repsm1 * (qv - qv0);
    b = g * (b - ((qli - qc0) - qi0));
    a.buoyancy[((size_t)(k + 1) * (nj + 6) + (jj + 3)) * (size_t)(ni + 6) + (ii + 3)] = b;
    a.thv[pp] = (theta * (1.0f + reps * qv)) / ((1.0f + qv) + qli);
    const float cpm = (cp + cpv * qv) + cpli;
    const float cvm = 1.0f / ((cv + cvv * qv) + cpli);
    a.thterm[cell] = (theta * ((rd + rv * qv) - rovcp * cpm)) * cvm;
    a.ppterm[pp] = (((bp + a.pp3d[pp]) * rovcp) * cpm) * cvm;
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" int32_t gm1b_eqtset2_stage_terms(int32_t ni, int32_t nj, int32_t nk, const gm1b_eqtset2_arrays *arrays,
                                           int32_t base3d, void *stream) {
    if (arrays == nullptr || ni < 1 || nj < 1 || nk < 1) {
        gm1b_set_error("gm1b_eqtset2_stage_terms: need arrays and ni, nj, nk >= 1");
        return GM1B_ERR_ARGUMENT;
    }
    const gm1b_eqtset2_arrays &a = *arrays;
    if (!a.th0 || !a.qv0 || !a.pi0 || !a.th3d || !a.q3d || !a.pp3d || !a.thv || !a.ppterm || !a.buoyancy ||
        !a.thterm || !a.piadv) {
        gm1b_set_error("gm1b_eqtset2_stage_terms: a required array is NULL (only qc0/qi0 may be)");
        return GM1B_ERR_ARGUMENT;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    ProfScope ps("eqtset2_terms_kernel", st);
    eqtset2_terms_kernel<<<dim3((ni + 2 + kBX - 1) / kBX, (nj + 2 + kBY - 1) / kBY, nk), dim3(kBX, kBY), 0, st>>>(
        a, ni, nj, nk, base3d ? 1 : 0);
    ps.stop();
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("eqtset2_terms_kernel: %s", cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}
