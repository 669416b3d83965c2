// tke.cu - sm_100a kernels of the Deardorff SGS/TKE local algebra: tkekm
// (grid scale, length scale, Km, Kh, dissipation), the free-slip lower face
// tkebc and the pre-turbt TKE source.
//
// Behaviour followed (reference file:line):
//   sgs_constants_f32    src/cm1core/cuda_sgs_tke.py:187-208
//   cpu_sgs_tke_inplace  src/cm1core/cuda_sgs_tke.py:220-357
//
// Design (B200): one elementwise pass over the w levels 1..nk-1 with x
// fastest (every array is (nk+1, nj, ni)), then a one-level pass for the
// lower face, which reads level 1's Km and Kh.
#include "gm1b_common.cuh"

namespace gm1b {
namespace {

constexpr int kSX = 32, kSY = 4;

struct SgsConst {
    float cme, ce1, ce2, csm;
};

__host__ SgsConst sgs_constants() {
    const float cme = 0.10f, c_l = 0.8165f, ri_c = 0.25f, pi = 3.1415926535897932384626433f;
    float ce1 = cme * c_l;
    ce1 = ce1 * c_l;
    ce1 = ce1 * (1.0f / ri_c - 1.0f);
    float ce2 = (cme * pi) * pi - ce1;
    ce2 = ce2 > 0.0f ? ce2 : 0.0f;
    const float numerator = (cme * cme) * cme;
    SgsConst c;
    c.cme = cme;
    c.ce1 = ce1;
    c.ce2 = ce2;
    c.csm = powf(numerator / (ce1 + ce2), 0.25f);
    return c;
}

// grid (ceil(ni/32), ceil(nj/4), nk-1): levels k = 1..nk-1
__global__ void __launch_bounds__(kSX *kSY)
    sgs_tke_kernel(gm1b_sgs_tke_arrays a, int ni, int nj, float dx, float dy, float dz, SgsConst c) {
    const int i = blockIdx.x * kSX + threadIdx.x;
    const int j = blockIdx.y * kSY + threadIdx.y;
    const int k = blockIdx.z + 1;
    if (i >= ni || j >= nj) return;
    const size_t p = ((size_t)k * nj + j) * (size_t)ni + i;
    const float c_l = 0.8165f, tke_min = 1.0e-10f, nm_min = 1.0e-6f, small = 0.001f;
    float grid = dx * a.ruh[i];
    grid = grid * (dy * a.rvh[j]);
    grid = grid * (dz * a.rmf[p]);
    grid = powf(grid, 0.33333333f);
    const float reciprocal = 1.0f / grid;
    const float nm = a.nm[p];
    const float tkea = a.tkea[p];
    float tk, length;
    if (tkea <= tke_min) {
        tk = tke_min;
        length = small * grid;
    } else {
        tk = tkea;
        length = grid;
        if (nm > nm_min) {
            length = c_l * sqrtf(tk / nm);
            length = fminf(length, grid);
            length = fmaxf(length, small * grid);
        }
    }
    a.grdscl[p] = grid;
    a.rgrdscl[p] = reciprocal;
    a.tk[p] = tk;
    a.lenscl[p] = length;
    a.cme[p] = c.cme;
    a.ce1[p] = c.ce1;
    a.ce2[p] = c.ce2;
    a.csm[p] = c.csm;
    const float sqrt_tk = sqrtf(tk);
    float df = c.ce2 * length;
    df = df * reciprocal;
    df = c.ce1 + df;
    float diss = df * tk;
    diss = diss * sqrt_tk;
    diss = diss / length;
    const float dissten = a.dissten[p] + diss;
    a.dissten[p] = dissten;
    float km = c.cme * sqrt_tk;
    km = km * length;
    a.kmh[p] = km;
    a.kmv[p] = km;
    float prinv = 3.0f;
    if (nm > nm_min) prinv = fminf(1.0f + 2.0f * (length * reciprocal), 3.0f);
    const float kh = km * prinv;
    a.khh[p] = kh;
    a.khv[p] = kh;
    float source = (-kh) * nm - dissten;
    const float deform = fmaxf(0.0f, a.defv[p] + a.defh[p]);
    source = source + km * deform;
    a.tketen[p] = source;
    if (a.clip_count != nullptr && tkea <= tke_min) atomicAdd(a.clip_count, 1u);
}

// free-slip lower face (tkebc), after level 1 is complete
__global__ void __launch_bounds__(kSX *kSY) sgs_tke_lower_face_kernel(gm1b_sgs_tke_arrays a, int ni, int nj) {
    const int i = blockIdx.x * kSX + threadIdx.x;
    const int j = blockIdx.y * kSY + threadIdx.y;
    if (i >= ni || j >= nj) return;
    const size_t p0 = (size_t)j * ni + i;
    const size_t p1 = (size_t)ni * nj + p0;
    a.tkea[p0] = 0.0f;
    const float kmh0 = 0.0f;
    a.kmh[p0] = kmh0;
    const float kmv0 = kmh0;
    a.kmv[p0] = kmv0;
    float ratio = a.khv[p1] / (1.0e-10f + a.kmv[p1]);
    a.khv[p0] = kmv0 * ratio;
    ratio = a.khh[p1] / (1.0e-10f + a.kmh[p1]);
    a.khh[p0] = kmh0 * ratio;
}

}  // namespace
}  // namespace gm1b

using namespace gm1b;

extern "C" int32_t gm1b_sgs_tke(int32_t ni, int32_t nj, int32_t nk, const gm1b_sgs_tke_arrays *arrays, float dx,
                               float dy, float dz, void *stream) {
    if (arrays == nullptr || ni < 1 || nj < 1 || nk < 2) {
        gm1b_set_error("gm1b_sgs_tke: need arrays, ni >= 1, nj >= 1, nk >= 2");
        return GM1B_ERR_ARGUMENT;
    }
    if (!(dx > 0.0f) || !(dy > 0.0f) || !(dz > 0.0f) || !isfinite(dx) || !isfinite(dy) || !isfinite(dz)) {
        gm1b_set_error("gm1b_sgs_tke: dx, dy, dz must be finite and > 0");
        return GM1B_ERR_ARGUMENT;
    }
    const float *const *p = reinterpret_cast<const float *const *>(arrays);
    for (size_t q = 0; q < 21; ++q)
        if (p[q] == nullptr) {
            gm1b_set_error("gm1b_sgs_tke: array #%zu is NULL", q);
            return GM1B_ERR_ARGUMENT;
        }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (arrays->clip_count != nullptr && cudaMemsetAsync(arrays->clip_count, 0, sizeof(uint32_t), st) != cudaSuccess) {
        gm1b_set_error("gm1b_sgs_tke: clip counter reset failed");
        return GM1B_ERR_CUDA;
    }
    const SgsConst c = sgs_constants();
    const dim3 blk(kSX, kSY);
    {
        ProfScope ps("sgs_tke_kernel", st);
        sgs_tke_kernel<<<dim3((ni + kSX - 1) / kSX, (nj + kSY - 1) / kSY, nk - 1), blk, 0, st>>>(*arrays, ni, nj, dx,
                                                                                                 dy, dz, c);
        ps.stop();
    }
    {
        ProfScope ps("sgs_tke_lower_face_kernel", st);
        sgs_tke_lower_face_kernel<<<dim3((ni + kSX - 1) / kSX, (nj + kSY - 1) / kSY), blk, 0, st>>>(*arrays, ni, nj);
        ps.stop();
    }
    cudaError_t e = cudaPeekAtLastError();
    if (e != cudaSuccess) {
        cudaGetLastError();
        gm1b_set_error("gm1b_sgs_tke: %s", cudaGetErrorString(e));
        return GM1B_ERR_CUDA;
    }
    return GM1B_OK;
}
