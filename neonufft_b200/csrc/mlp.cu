// Multilayer perceptron kernels for the engine's learned cost model (FP32).
//
// No counterpart in the reference. The tuner (neonufft_b200/tuner.py) predicts the run time of
// a transform configuration with a small MLP trained on timings the engine itself measures;
// its forward pass, backward pass, loss gradient and Adam update run here.
//
// Network: L weight layers, widths w_0 (inputs) .. w_L (outputs); hidden layers tanh, output
// linear. Parameters, per layer l = 1..L in order: W_l (w_l x w_{l-1}, row-major) then b_l
// (w_l). Activations are kept per layer, batch-major (A_l[b * w_l + j]), in one workspace of
// sum_{l>=1} w_l * batch floats; the network output is the last block. The layers are a few
// dozen wide, so every kernel is a plain one-thread-per-output loop; sums run in a fixed order,
// so results do not depend on the launch.
#include <cmath>
#include <vector>

#include "kernels.cuh"

namespace nnb {

namespace {

constexpr int kMlpThreads = 256;

unsigned blocks_for(i64 n) { return unsigned((n + kMlpThreads - 1) / kMlpThreads); }

// A[b, j] = act(sum_i W[j, i] X[b, i] + bias[j])
__global__ void __launch_bounds__(kMlpThreads)
    dense_forward_kernel(const float* W, const float* bias, const float* X, i64 batch, int nin,
                         int nout, int tanh_act, float* A) {
  const i64 t = blockIdx.x * i64(kMlpThreads) + threadIdx.x;
  if (t >= batch * nout) return;
  const i64 b = t / nout;
  const int j = int(t - b * nout);
  const float* w = W + i64(j) * nin;
  const float* x = X + b * nin;
  float z = bias[j];
  for (int i = 0; i < nin; ++i) z = fmaf(w[i], x[i], z);
  A[t] = tanh_act ? tanhf(z) : z;
}

// dZ = dA * act'(Z), in place (tanh' = 1 - A^2).
__global__ void __launch_bounds__(kMlpThreads)
    act_backward_kernel(const float* A, i64 n, int tanh_act, float* dA) {
  const i64 t = blockIdx.x * i64(kMlpThreads) + threadIdx.x;
  if (t >= n || !tanh_act) return;
  dA[t] *= 1.f - A[t] * A[t];
}

// gW[j, i] = sum_b dZ[b, j] X[b, i]; gb[j] = sum_b dZ[b, j]
__global__ void __launch_bounds__(kMlpThreads)
    dense_grad_kernel(const float* dZ, const float* X, i64 batch, int nin, int nout, float* gW,
                      float* gb) {
  const i64 t = blockIdx.x * i64(kMlpThreads) + threadIdx.x;
  const i64 nw = i64(nout) * nin;
  if (t < nw) {
    const int j = int(t / nin);
    const int i = int(t - i64(j) * nin);
    float s = 0.f;
    for (i64 b = 0; b < batch; ++b) s = fmaf(dZ[b * nout + j], X[b * nin + i], s);
    gW[t] = s;
  } else if (t < nw + nout) {
    const int j = int(t - nw);
    float s = 0.f;
    for (i64 b = 0; b < batch; ++b) s += dZ[b * nout + j];
    gb[j] = s;
  }
}

// dX[b, i] = sum_j W[j, i] dZ[b, j]
__global__ void __launch_bounds__(kMlpThreads)
    dense_input_grad_kernel(const float* W, const float* dZ, i64 batch, int nin, int nout,
                            float* dX) {
  const i64 t = blockIdx.x * i64(kMlpThreads) + threadIdx.x;
  if (t >= batch * nin) return;
  const i64 b = t / nin;
  const int i = int(t - b * nin);
  float s = 0.f;
  for (int j = 0; j < nout; ++j) s = fmaf(W[i64(j) * nin + i], dZ[b * nout + j], s);
  dX[t] = s;
}

// dy = 2 (y - target) / n; loss (one float, zeroed by the host launcher) += (y - target)^2 / n
__global__ void __launch_bounds__(kMlpThreads)
    mse_kernel(const float* y, const float* target, i64 n, float* dy, float* loss) {
  const i64 t = blockIdx.x * i64(kMlpThreads) + threadIdx.x;
  float e2 = 0.f;
  if (t < n) {
    const float e = y[t] - target[t];
    dy[t] = 2.f * e / float(n);
    e2 = e * e / float(n);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e2 += __shfl_xor_sync(0xffffffffu, e2, o);
  if ((threadIdx.x & 31) == 0 && e2 != 0.f) atomicAdd(loss, e2);
}

__global__ void __launch_bounds__(kMlpThreads)
    adam_kernel(i64 n, float* p, const float* g, float* m, float* v, float lr, float b1,
                float b2, float eps, float c1, float c2) {
  const i64 t = blockIdx.x * i64(kMlpThreads) + threadIdx.x;
  if (t >= n) return;
  const float gt = g[t];
  const float mt = b1 * m[t] + (1.f - b1) * gt;
  const float vt = b2 * v[t] + (1.f - b2) * gt * gt;
  m[t] = mt;
  v[t] = vt;
  p[t] -= lr * (mt / c1) / (sqrtf(vt / c2) + eps);
}

void check_widths(int L, const int* widths) {
  if (L < 1 || L > 16 || !widths) throw_input("an MLP has 1 to 16 layers");
  for (int l = 0; l <= L; ++l) {
    if (widths[l] < 1 || widths[l] > 4096) throw_input("MLP layer widths must be in [1, 4096]");
  }
}

}  // namespace

i64 mlp_param_count(int L, const int* widths) {
  check_widths(L, widths);
  i64 n = 0;
  for (int l = 1; l <= L; ++l) n += i64(widths[l]) * widths[l - 1] + widths[l];
  return n;
}

void mlp_forward(int L, const int* widths, const float* params, const float* x, i64 batch,
                 float* acts, cudaStream_t stream) {
  check_widths(L, widths);
  if (batch <= 0) return;
  const float* in = x;
  const float* p = params;
  float* a = acts;
  for (int l = 1; l <= L; ++l) {
    const int nin = widths[l - 1], nout = widths[l];
    dense_forward_kernel<<<blocks_for(batch * nout), kMlpThreads, 0, stream>>>(
        p, p + i64(nout) * nin, in, batch, nin, nout, l < L ? 1 : 0, a);
    NNB_LAUNCH_CHECK();
    p += i64(nout) * nin + nout;
    in = a;
    a += batch * nout;
  }
}

void mlp_backward(int L, const int* widths, const float* params, const float* x,
                  const float* acts, float* dacts, i64 batch, float* grads,
                  cudaStream_t stream) {
  check_widths(L, widths);
  if (batch <= 0) return;
  std::vector<i64> poff(size_t(L + 1)), aoff(size_t(L + 1));
  poff[0] = 0;
  aoff[0] = 0;
  for (int l = 1; l <= L; ++l) {
    poff[size_t(l)] = poff[size_t(l - 1)] + i64(widths[l]) * widths[l - 1] + widths[l];
    aoff[size_t(l)] = aoff[size_t(l - 1)] + batch * widths[l];
  }
  for (int l = L; l >= 1; --l) {
    const int nin = widths[l - 1], nout = widths[l];
    const float* A = acts + aoff[size_t(l - 1)];
    float* dZ = dacts + aoff[size_t(l - 1)];
    const float* X = l > 1 ? acts + aoff[size_t(l - 2)] : x;
    act_backward_kernel<<<blocks_for(batch * nout), kMlpThreads, 0, stream>>>(
        A, batch * nout, l < L ? 1 : 0, dZ);
    NNB_LAUNCH_CHECK();
    float* gW = grads + poff[size_t(l - 1)];
    dense_grad_kernel<<<blocks_for(i64(nout) * nin + nout), kMlpThreads, 0, stream>>>(
        dZ, X, batch, nin, nout, gW, gW + i64(nout) * nin);
    NNB_LAUNCH_CHECK();
    if (l > 1) {
      dense_input_grad_kernel<<<blocks_for(batch * nin), kMlpThreads, 0, stream>>>(
          params + poff[size_t(l - 1)], dZ, batch, nin, nout, dacts + aoff[size_t(l - 2)]);
      NNB_LAUNCH_CHECK();
    }
  }
}

void mlp_mse(const float* y, const float* target, i64 n, float* dy, float* loss,
             cudaStream_t stream) {
  if (n <= 0) return;
  NNB_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), stream));
  mse_kernel<<<blocks_for(n), kMlpThreads, 0, stream>>>(y, target, n, dy, loss);
  NNB_LAUNCH_CHECK();
}

void mlp_adam(i64 n, float* params, const float* grads, float* m, float* v, float lr,
              float beta1, float beta2, float eps, i64 step, cudaStream_t stream) {
  if (n <= 0) return;
  if (step < 1) throw_input("Adam steps count from 1");
  const float c1 = 1.f - std::pow(beta1, float(step));
  const float c2 = 1.f - std::pow(beta2, float(step));
  adam_kernel<<<blocks_for(n), kMlpThreads, 0, stream>>>(n, params, grads, m, v, lr, beta1,
                                                         beta2, eps, c1, c2);
  NNB_LAUNCH_CHECK();
}

}  // namespace nnb
