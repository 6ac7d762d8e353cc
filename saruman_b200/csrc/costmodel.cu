// costmodel.cu -- forward, backward and Adam kernels of the autotuner's
// cost model: a small fully connected network (tanh hidden layers, linear
// output) that predicts the banded kernel's log time per candidate from a
// bin's features and a launch shape.  fp32 throughout; every reduction runs
// in a fixed order (one thread per output, a sequential loop over the
// samples), so gradients are deterministic and comparable with a CPU
// reference.
//
// Parameter layout (one float array): for each layer l with fan-in a and
// fan-out b, W_l (b x a, row-major) then bias_l (b).  Work layout: for each
// layer the activations H_l (n x b), then one gradient buffer per layer of
// the same shape.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "../../include/saruman_b200.h"
#include "server_internal.h"

namespace {

constexpr int kMaxLayers = 8;
constexpr int kMaxWidth = 1024;

struct Net {
  int nl = 0;                  // weight layers
  int dims[kMaxLayers + 1]{};  // dims[0] = features, dims[nl] = 1
  long w_off[kMaxLayers]{}, b_off[kMaxLayers]{};
  long params = 0;
};

bool make_net(const int32_t *dims, int32_t nlayers, Net *net) {
  if (!dims || nlayers < 1 || nlayers > kMaxLayers) return false;
  net->nl = nlayers;
  long off = 0;
  for (int l = 0; l <= nlayers; ++l) {
    if (dims[l] < 1 || dims[l] > kMaxWidth) return false;
    net->dims[l] = dims[l];
  }
  for (int l = 0; l < nlayers; ++l) {
    net->w_off[l] = off;
    off += (long)dims[l + 1] * dims[l];
    net->b_off[l] = off;
    off += dims[l + 1];
  }
  net->params = off;
  return true;
}

long act_floats(const Net &net, long n) {  // activations of every layer
  long t = 0;
  for (int l = 1; l <= net.nl; ++l) t += n * net.dims[l];
  return t;
}

// h_out[i][j] = act(b[j] + sum_c W[j][c] h_in[i][c]); tanh unless last layer
__global__ void dense_forward(const float *__restrict__ W, const float *__restrict__ bias,
                              const float *__restrict__ h_in, float *__restrict__ h_out, int n,
                              int fan_in, int fan_out, int linear) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)n * fan_out) return;
  const int i = (int)(idx / fan_out), j = (int)(idx % fan_out);
  float z = bias[j];
  const float *w = W + (long)j * fan_in;
  const float *h = h_in + (long)i * fan_in;
  for (int c = 0; c < fan_in; ++c) z = fmaf(w[c], h[c], z);
  h_out[idx] = linear ? z : tanhf(z);
}

// delta of the linear output for the mean squared error: 2 (p - y) / n
__global__ void mse_delta(const float *__restrict__ pred, const float *__restrict__ y,
                          float *__restrict__ delta, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) delta[i] = 2.0f * (pred[i] - y[i]) / (float)n;
}

// loss = mean (p - y)^2, one block, fixed reduction order
__global__ void mse_loss(const float *__restrict__ pred, const float *__restrict__ y,
                         float *__restrict__ loss, int n) {
  __shared__ float part[256];
  float s = 0.f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const float d = pred[i] - y[i];
    s = fmaf(d, d, s);
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int w = blockDim.x / 2; w > 0; w >>= 1) {
    if ((int)threadIdx.x < w) part[threadIdx.x] += part[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss = part[0] / (float)n;
}

// gW[j][c] = sum_i delta[i][j] h_in[i][c];  gb[j] = sum_i delta[i][j]
__global__ void dense_weight_grad(const float *__restrict__ delta, const float *__restrict__ h_in,
                                  float *__restrict__ gW, float *__restrict__ gb, int n,
                                  int fan_in, int fan_out) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nw = (long)fan_out * fan_in;
  if (idx < nw) {
    const int j = (int)(idx / fan_in), c = (int)(idx % fan_in);
    float s = 0.f;
    for (int i = 0; i < n; ++i) s = fmaf(delta[(long)i * fan_out + j], h_in[(long)i * fan_in + c], s);
    gW[idx] = s;
  } else if (idx < nw + fan_out) {
    const int j = (int)(idx - nw);
    float s = 0.f;
    for (int i = 0; i < n; ++i) s += delta[(long)i * fan_out + j];
    gb[j] = s;
  }
}

// delta_in[i][c] = (sum_j W[j][c] delta[i][j]) * (1 - h_in[i][c]^2)  (tanh')
__global__ void dense_input_grad(const float *__restrict__ W, const float *__restrict__ delta,
                                 const float *__restrict__ h_in, float *__restrict__ delta_in,
                                 int n, int fan_in, int fan_out) {
  const long idx = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (long)n * fan_in) return;
  const int i = (int)(idx / fan_in), c = (int)(idx % fan_in);
  float s = 0.f;
  for (int j = 0; j < fan_out; ++j) s = fmaf(W[(long)j * fan_in + c], delta[(long)i * fan_out + j], s);
  const float h = h_in[idx];
  delta_in[idx] = s * (1.0f - h * h);
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g,
                            float *__restrict__ m, float *__restrict__ v, long count, float lr,
                            float b1, float b2, float eps, float c1, float c2) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

unsigned blocks_for(long threads) { return (unsigned)((threads + 255) / 256); }

// forward over all layers; activations of layer l at act + act_off[l]
cudaError_t forward(const Net &net, const float *params, const float *x, int n, float *act,
                    cudaStream_t s) {
  const float *h = x;
  float *out = act;
  for (int l = 0; l < net.nl; ++l) {
    const int a = net.dims[l], b = net.dims[l + 1];
    dense_forward<<<blocks_for((long)n * b), 256, 0, s>>>(params + net.w_off[l],
                                                         params + net.b_off[l], h, out, n, a, b,
                                                         l == net.nl - 1);
    h = out;
    out += (long)n * b;
  }
  return cudaGetLastError();
}

int check(const Net &net, int32_t n) {
  if (n < 1 || net.dims[net.nl] != 1) {
    saru::set_last_error("cost model: n >= 1 and one output");
    return SARU_E_INVALID;
  }
  return SARU_OK;
}

}  // namespace

extern "C" {

int64_t saru_mlp_param_count(const int32_t *dims, int32_t nlayers) {
  Net net;
  return make_net(dims, nlayers, &net) ? net.params : -1;
}

int64_t saru_mlp_work_floats(const int32_t *dims, int32_t nlayers, int32_t n) {
  Net net;
  if (!make_net(dims, nlayers, &net) || n < 1) return -1;
  return 2 * act_floats(net, n) + 1;  // activations, deltas, loss
}

int saru_mlp_forward(const int32_t *dims, int32_t nlayers, const float *params, const float *x,
                     int32_t n, float *y, float *work, void *stream) {
  Net net;
  if (!make_net(dims, nlayers, &net)) {
    saru::set_last_error("cost model: 1..8 layers of width 1..1024");
    return SARU_E_INVALID;
  }
  if (int rc = check(net, n)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t e = forward(net, params, x, n, work, s);
  const long last = act_floats(net, n) - n;
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(y, work + last, sizeof(float) * (size_t)n, cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) {
    saru::set_last_error(cudaGetErrorString(e));
    return SARU_E_CUDA;
  }
  saru::count_launch();
  return SARU_OK;
}

int saru_mlp_loss_grad(const int32_t *dims, int32_t nlayers, const float *params, const float *x,
                       const float *y, int32_t n, float *loss, float *grad, float *work,
                       void *stream) {
  Net net;
  if (!make_net(dims, nlayers, &net)) {
    saru::set_last_error("cost model: 1..8 layers of width 1..1024");
    return SARU_E_INVALID;
  }
  if (int rc = check(net, n)) return rc;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  float *act = work;
  float *dlt = work + act_floats(net, n);
  cudaError_t e = forward(net, params, x, n, act, s);
  // offsets of each layer's activations / deltas
  long off[kMaxLayers + 1];
  off[0] = 0;
  for (int l = 1; l <= net.nl; ++l) off[l] = off[l - 1] + (long)n * net.dims[l];
  const float *pred = act + off[net.nl - 1];
  float *d_out = dlt + off[net.nl - 1];
  if (e == cudaSuccess) {
    mse_loss<<<1, 256, 0, s>>>(pred, y, loss, n);
    mse_delta<<<blocks_for(n), 256, 0, s>>>(pred, y, d_out, n);
    e = cudaGetLastError();
  }
  for (int l = net.nl - 1; l >= 0 && e == cudaSuccess; --l) {
    const int a = net.dims[l], b = net.dims[l + 1];
    const float *h_in = l ? act + off[l - 1] : x;
    const float *d = dlt + off[l];
    dense_weight_grad<<<blocks_for((long)b * a + b), 256, 0, s>>>(
        d, h_in, grad + net.w_off[l], grad + net.b_off[l], n, a, b);
    if (l > 0)
      dense_input_grad<<<blocks_for((long)n * a), 256, 0, s>>>(params + net.w_off[l], d, h_in,
                                                               dlt + off[l - 1], n, a, b);
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    saru::set_last_error(cudaGetErrorString(e));
    return SARU_E_CUDA;
  }
  saru::count_launch();
  return SARU_OK;
}

int saru_mlp_adam_step(float *params, const float *grad, float *m, float *v, int64_t count,
                       float lr, float beta1, float beta2, float eps, int32_t step,
                       void *stream) {
  if (count < 1 || step < 1) {
    saru::set_last_error("saru_mlp_adam_step: count >= 1 and step >= 1");
    return SARU_E_INVALID;
  }
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam_kernel<<<blocks_for(count), 256, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      params, grad, m, v, count, lr, beta1, beta2, eps, c1, c2);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    saru::set_last_error(cudaGetErrorString(e));
    return SARU_E_CUDA;
  }
  saru::count_launch();
  return SARU_OK;
}

}  // extern "C"
