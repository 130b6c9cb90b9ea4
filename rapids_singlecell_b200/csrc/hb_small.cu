// Kernel-level entry points on the small [B, K] tables (penalty, ridge lambda,
// arrowhead inverse).  Inside hb_harmonize these steps are fused into the block
// update and the ridge solve; they are exported separately so the reference's
// per-kernel known-answer tests can be run against this engine.
#include "hb_internal.h"

namespace hb {

__global__ void k_penalty(const double* __restrict__ E, const double* __restrict__ O,
                          const double* __restrict__ theta, double* __restrict__ pen, int B, int K,
                          int stabilized) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * K) return;
  const int b = i / K;
  const double denom = stabilized ? (O[i] + E[i] + 1.0) : (O[i] + 1.0);
  pen[i] = pow((E[i] + 1.0) / denom, theta[b]);
}

__global__ void k_lambda_kb(const double* __restrict__ E, const double* __restrict__ O,
                            const double* __restrict__ Nb, double* __restrict__ lam, int B, int K,
                            double alpha, double threshold, int prune, double ridge_lambda,
                            int dynamic_lambda) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= B * K) return;
  const int b = i / K;
  double l;
  if (!dynamic_lambda) {
    l = ridge_lambda;
  } else {
    l = alpha * E[i];
    if (prune) {
      const double nb = Nb[b];
      const double safe = nb > 0 ? nb : 1.0;
      if (O[i] / safe < threshold || nb == 0) l = 1e30;
    }
  }
  if (O[i] + l == 0.0) l = 1e30;
  lam[i] = l;
}

__global__ void k_ridge_inverse(const double* __restrict__ O, const double* __restrict__ lam,
                                double* __restrict__ inv, int B, int K) {
  extern __shared__ double sh[];
  double* f = sh;
  double* p = sh + B;
  __shared__ double red[32];
  const int k = blockIdx.x;
  double nk = 0, cneg = 0;
  for (int b = threadIdx.x; b < B; b += blockDim.x) {
    const double o = O[(size_t)b * K + k];
    const double fb = 1.0 / (o + lam[(size_t)b * K + k]);
    f[b] = fb;
    p[b] = -fb * o;
    nk += o;
    cneg += fb * o * o;
  }
  nk = block_sum(nk, red);
  cneg = block_sum(cneg, red);
  const double cinv = 1.0 / (nk - cneg);
  const int nb1 = B + 1;
  double* out = inv + (size_t)k * nb1 * nb1;
  for (int e = threadIdx.x; e < nb1 * nb1; e += blockDim.x) {
    const int i = e / nb1, j = e % nb1;
    double v;
    if (i == 0 && j == 0) v = cinv;
    else if (i == 0) v = cinv * p[j - 1];
    else if (j == 0) v = p[i - 1] * cinv;
    else {
      v = p[i - 1] * cinv * p[j - 1];
      if (i == j) v += f[i - 1];
    }
    out[e] = v;
  }
}

}  // namespace hb

using namespace hb;

extern "C" {

int hb_penalty(const double* E, const double* O, const double* theta, double* penalty,
               int32_t n_batches, int32_t n_clusters, int32_t stabilized, void* stream) {
  const int tot = n_batches * n_clusters;
  if (tot <= 0) return HB_OK;
  k_penalty<<<div_up(tot, 256), 256, 0, (cudaStream_t)stream>>>(E, O, theta, penalty, n_batches,
                                                                n_clusters, stabilized);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

int hb_lambda_kb(const double* E, const double* O, const double* N_b, double* lambda_kb,
                 int32_t n_batches, int32_t n_clusters, double alpha, double threshold,
                 int32_t prune, double ridge_lambda, int32_t dynamic_lambda, void* stream) {
  const int tot = n_batches * n_clusters;
  if (tot <= 0) return HB_OK;
  k_lambda_kb<<<div_up(tot, 256), 256, 0, (cudaStream_t)stream>>>(
      E, O, N_b, lambda_kb, n_batches, n_clusters, alpha, threshold, prune, ridge_lambda,
      dynamic_lambda);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

int hb_ridge_inverse(const double* O, const double* lambda_kb, double* inv, int32_t n_batches,
                     int32_t n_clusters, void* stream) {
  if (n_batches < 1 || n_clusters < 1) { set_error("bad shape"); return HB_ERR_INVALID; }
  k_ridge_inverse<<<n_clusters, 128, sizeof(double) * 2 * n_batches, (cudaStream_t)stream>>>(
      O, lambda_kb, inv, n_batches, n_clusters);
  HB_LAUNCH_CHECK();
  return HB_OK;
}

}  // extern "C"
