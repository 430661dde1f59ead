// ens_stats.cu -- ensemble mean and spread of the state fields (the output
// statistics after the analysis: ensemble_mesp, letkf/run/src/common.f90:
// 505-596, written as the mean / spread files by write_ens_mpi,
// common_io.f90:863-1009).
//
// One thread per (variable, level, column), columns fastest so a warp reads
// 32 consecutive values of each member: every state value is read once
// (HBM-bound, 4 or 8 bytes per member per point).  The sums are FP64 and
// shifted by the first member, d = x_m - x_1:
//   mean = x_1 + sum(d)/k,  spread = sqrt((sum(d^2) - sum(d)^2/k) / (k-1)),
// the one-pass form of the reference's two-pass mean and (k-1) spread.
#include "internal.cuh"

namespace sbl {
namespace {

template <typename ST>
__global__ void k_ens_mesp(long long npts, long long stride_m, long long per_var, int k, const ST *__restrict__ x,
                           ST *__restrict__ mean, ST *__restrict__ sprd) {
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < npts; t += (long long)gridDim.x * blockDim.x) {
    const long long v = t / per_var, r = t - v * per_var;      // r = level * ncol + column
    const ST *xv = x + v * (long long)k * stride_m + r;
    const double x1 = (double)xv[0];
    double s1 = 0.0, s2 = 0.0;
    for (int m = 1; m < k; ++m) {
      const double d = (double)xv[(long long)m * stride_m] - x1;
      s1 += d;
      s2 = fma(d, d, s2);
    }
    mean[t] = (ST)(x1 + s1 / (double)k);
    if (sprd) {
      const double nan = __longlong_as_double(0x7ff8000000000000LL);  // undef for k = 1
      sprd[t] = (ST)(k > 1 ? sqrt(fmax(s2 - s1 * s1 / (double)k, 0.0) / (double)(k - 1)) : nan);
    }
  }
}

template <typename ST>
int launch_t(const sbletkf_params *p, int nij1, const void *s3, const void *s2, void *m3, void *sd3, void *m2,
             void *sd2, cudaStream_t s) {
  int dev = 0, nsm = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int tb = 256;
  const long long ncol = nij1;
  if (p->nv3d > 0) {
    const long long n = (long long)p->nv3d * p->nlev * ncol;
    const long long nb = (n + tb - 1) / tb;
    const unsigned g = (unsigned)(nb < (long long)nsm * 16 ? nb : (long long)nsm * 16);
    k_ens_mesp<ST><<<g, tb, 0, s>>>(n, (long long)p->nlev * ncol, (long long)p->nlev * ncol, p->nmem,
                                     (const ST *)s3, (ST *)m3, (ST *)sd3);
  }
  if (p->nv2d > 0) {
    const long long n = (long long)p->nv2d * ncol;
    const long long nb = (n + tb - 1) / tb;
    const unsigned g = (unsigned)(nb < (long long)nsm * 16 ? nb : (long long)nsm * 16);
    k_ens_mesp<ST><<<g, tb, 0, s>>>(n, ncol, ncol, p->nmem, (const ST *)s2, (ST *)m2, (ST *)sd2);
  }
  return cuda_status(cudaGetLastError());
}

}  // namespace

int launch_ens_mesp(const sbletkf_params *p, int nij1, const void *s3, const void *s2, int dtype, void *m3, void *sd3,
                    void *m2, void *sd2, cudaStream_t s) {
  if (dtype == SBLETKF_F64) return launch_t<double>(p, nij1, s3, s2, m3, sd3, m2, sd2, s);
  return launch_t<float>(p, nij1, s3, s2, m3, sd3, m2, sd2, s);
}

}  // namespace sbl
