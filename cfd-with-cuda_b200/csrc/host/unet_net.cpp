// U-Net parameter handling and forward / backward / Adam drivers.
#include "unet_net.h"

#include <cmath>
#include <cstdlib>
#include <cstring>


namespace cfd {

const UnetTensorSpec kUnetTensor[kUnetTensors] = {
    {0, 1},  {0, 16}, {1, 32}, {1, 32}, {2, 64}, {2, 64}, {2, 64},
    {2, 32}, {1, 32}, {1, 32}, {1, 16}, {0, 16}, {0, 16}, {0, 1},
};
const UnetConvSpec kUnetConv[kUnetConvs] = {
    {0, 1, 1, 1},  {1, 2, 2, 1},  {2, 3, 1, 1},   {3, 4, 2, 1},   {4, 5, 1, 1},  {5, 6, 1, 1},
    {6, 7, 1, 1},  {8, 9, 1, 1},  {9, 10, 1, 1},  {11, 12, 1, 1}, {12, 13, 1, 0},
};
const UnetUpSpec kUnetUp[2] = {{7, 3, 8}, {10, 1, 11}};

namespace {

// Execution order: conv index >= 0, prolongation -1 - index.
const int kOrder[kUnetConvs + 2] = {0, 1, 2, 3, 4, 5, 6, -1, 7, 8, -2, 9, 10};

long long wcount(int l) {
  return 27LL * kUnetTensor[kUnetConv[l].in].ch * kUnetTensor[kUnetConv[l].out].ch;
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}
double uniform01(uint64_t& s) { return ((splitmix(s) >> 11) + 0.5) * (1.0 / 9007199254740992.0); }

template <class T>
cudaError_t grow(T*& p, long long& cap, long long n, int* gen = nullptr) {
  if (n <= cap) return cudaSuccess;
  if (gen) ++*gen;
  if (p) cudaFree(p);
  p = nullptr;
  cap = 0;
  cudaError_t e = cudaMalloc((void**)&p, (size_t)n * sizeof(T));
  if (e == cudaSuccess) cap = n;
  return e;
}

}  // namespace

long long unet_param_count() {
  long long n = 0;
  for (int l = 0; l < kUnetConvs; l++) n += wcount(l) + kUnetTensor[kUnetConv[l].out].ch;
  return n;
}
long long unet_weight_offset(int layer) {
  long long n = 0;
  for (int l = 0; l < layer; l++) n += wcount(l) + kUnetTensor[kUnetConv[l].out].ch;
  return n;
}
long long unet_bias_offset(int layer) { return unet_weight_offset(layer) + wcount(layer); }

UnetNet::~UnetNet() {
  cudaFree(P);
  cudaFree(G);
  cudaFree(M1);
  cudaFree(M2);
  cudaFree(Pb);
  for (int t = 0; t < kUnetTensors; t++) {
    cudaFree(act[t]);
    cudaFree(grad[t]);
  }
  cudaFree(out);
  cudaFree(lossv);
  cudaFree(tc_err);
  for (int l = 0; l < kUnetConvs; l++) {
    cudaFree(wpack[l]);
  }
  if (h_pinned) cudaFreeHost(h_pinned);
  if (own_stream) cudaStreamDestroy(own_stream);
}

int UnetNet::init(unsigned long long seed) {
  nparam = unet_param_count();
  if (cudaGetDevice(&device) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&num_sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || num_sms < 1) {
    err = "cannot read the SM count of the device";
    return -1;
  }
  if (const char* e = std::getenv("CFD_UNET_TC")) tc_enabled = std::atoi(e) != 0;
  if (const char* e = std::getenv("CFD_CONV_PIPE")) conv_pipe = std::atoi(e);
  if (!own_stream && cudaStreamCreateWithFlags(&own_stream, cudaStreamNonBlocking) != cudaSuccess) return -1;
  const size_t b = (size_t)nparam * sizeof(float);
  if (cudaMalloc((void**)&P, b) || cudaMalloc((void**)&G, b) || cudaMalloc((void**)&M1, b) ||
      cudaMalloc((void**)&M2, b) || cudaMalloc((void**)&Pb, (size_t)nparam * sizeof(__nv_bfloat16)) ||
      cudaMalloc((void**)&lossv, 64 * sizeof(float)) || cudaMallocHost((void**)&h_pinned, 64 * sizeof(float)) ||
      cudaMalloc((void**)&tc_err, sizeof(int)) || cudaMemset(tc_err, 0, sizeof(int))) {
    err = "U-Net parameter allocation failed";
    return -1;
  }
  // He-normal weights for the leaky-ReLU layers (Box-Muller on a splitmix64
  // stream, so the same seed gives the same network on every platform), a
  // ten times smaller scale on the output layer, zero biases.
  std::vector<float> h((size_t)nparam, 0.f);
  uint64_t st = seed;
  for (int l = 0; l < kUnetConvs; l++) {
    const int cin = kUnetTensor[kUnetConv[l].in].ch;
    double sd = std::sqrt(2.0 / ((1.0 + kLeaky * kLeaky) * 27.0 * cin));
    if (!kUnetConv[l].act) sd = 0.1 * std::sqrt(1.0 / (27.0 * cin));
    const long long w0 = unet_weight_offset(l);
    for (long long i = 0; i < wcount(l); i++) {
      const double u1 = uniform01(st), u2 = uniform01(st);
      h[(size_t)(w0 + i)] = (float)(sd * std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2));
    }
  }
  return set_params(h.data(), nparam);
}

int UnetNet::set_params(const float* h, long long n) {
  if (n != nparam) {
    err = "parameter count mismatch";
    return -1;
  }
  cudaStream_t s = own_stream;
  if (cudaMemcpyAsync(P, h, (size_t)n * sizeof(float), cudaMemcpyHostToDevice, s) ||
      cudaMemsetAsync(M1, 0, (size_t)n * sizeof(float), s) || cudaMemsetAsync(M2, 0, (size_t)n * sizeof(float), s) ||
      cudaMemsetAsync(G, 0, (size_t)n * sizeof(float), s) || f32_to_bf16(n, P, Pb, s) ||
      cudaStreamSynchronize(s)) {
    err = "parameter upload failed";
    return -1;
  }
  launches++;
  adam_t = 0;
  packs_dirty = true;
  return 0;
}

int UnetNet::get_params(float* h, long long n) {
  if (n != nparam) {
    err = "parameter count mismatch";
    return -1;
  }
  if (cudaMemcpy(h, P, (size_t)n * sizeof(float), cudaMemcpyDeviceToHost)) {
    err = "parameter download failed";
    return -1;
  }
  return 0;
}

int UnetNet::set_grid(const int d[3], bool train) {
  for (int a = 0; a < 3; a++) {
    if (d[a] < 5 || (d[a] - 1) % 4 != 0) {
      err = "U-Net grid needs (n - 1) % 4 == 0 and n >= 5 on every axis";
      return -1;
    }
    dims[0][a] = d[a];
    dims[1][a] = (d[a] - 1) / 2 + 1;
    dims[2][a] = (dims[1][a] - 1) / 2 + 1;
  }
  for (int l = 0; l < 3; l++) nvox[l] = (long long)dims[l][0] * dims[l][1] * dims[l][2];
  cudaError_t e = cudaSuccess;
  for (int t = 0; t < kUnetTensors - 1 && e == cudaSuccess; t++)
    e = grow(act[t], cap[t], nvox[kUnetTensor[t].level] * kUnetTensor[t].ch, &gen);
  if (e == cudaSuccess) e = grow(out, out_cap, nvox[0], &gen);
  for (int t = 1; train && t < kUnetTensors && e == cudaSuccess; t++)
    e = grow(grad[t], gcap[t], nvox[kUnetTensor[t].level] * kUnetTensor[t].ch);
  if (e != cudaSuccess) {
    err = std::string("U-Net activation allocation: ") + cudaGetErrorString(e);
    return -1;
  }
  return 0;
}

namespace {

ConvDesc conv_desc(const UnetNet& n, int l, float* out_f32, const int* skip = nullptr) {
  const UnetConvSpec& c = kUnetConv[l];
  ConvDesc d{};
  const int li = kUnetTensor[c.in].level, lo = kUnetTensor[c.out].level;
  for (int a = 0; a < 3; a++) {
    d.in_dims[a] = n.dims[li][a];
    d.out_dims[a] = n.dims[lo][a];
  }
  d.stride = c.stride;
  d.inA = n.act[c.in];
  d.ca = kUnetTensor[c.in].ch;
  d.inB = nullptr;
  d.cb = 0;
  d.cout = kUnetTensor[c.out].ch;
  d.w = n.Pb + unet_weight_offset(l);
  d.bias = n.P + unet_bias_offset(l);
  if (c.out == kUnetTensors - 1) {
    d.out = nullptr;
    d.out_f32 = out_f32;
  } else {
    d.out = n.act[c.out];
    d.out_f32 = nullptr;
  }
  d.act = c.act;
  d.skip = skip;
  return d;
}

}  // namespace

cudaError_t UnetNet::prepare_tc(cudaStream_t s) {
  if (packs_dirty) {
    for (int l = 0; l < kUnetConvs; l++) {
      const int cin = kUnetTensor[kUnetConv[l].in].ch, cout = kUnetTensor[kUnetConv[l].out].ch;
      const int st = kUnetConv[l].stride;
      if (cin % 16) continue;
      cudaError_t e = grow(wpack[l], wpack_cap[l], conv_tc_pack_elems(cin, cout, st));
      if (e == cudaSuccess) e = conv_tc_pack(Pb + unet_weight_offset(l), cin, cout, st, wpack[l], s, pipe_mode(st) == 2);
      launches++;
      if (e != cudaSuccess) return e;
    }
    packs_dirty = false;
  }
  if (plan_gen != gen || plan_dims[0] != dims[0][0] || plan_dims[1] != dims[0][1] || plan_dims[2] != dims[0][2]) {
    for (int l = 0; l < kUnetConvs; l++) {
      ConvDesc d = conv_desc(*this, l, out);
      plan_ok[l] = false;
      if (!wpack[l] || !conv_tc_supported(d)) continue;
      plan_ok[l] = conv_tc_plan(d, wpack[l], num_sms, plans[l], pipe_mode(d.stride)) == 0;
    }
    plan_gen = gen;
    for (int a = 0; a < 3; a++) plan_dims[a] = dims[0][a];
  }
  return cudaSuccess;
}

cudaError_t UnetNet::forward(cudaStream_t s, float* out_f32, const int* skip) {
  if (!out_f32) out_f32 = out;
  if (tc_enabled) {
    cudaError_t e = prepare_tc(s);
    if (e != cudaSuccess) return e;
  }
  for (int op : kOrder) {
    cudaError_t e;
    if (op >= 0) {
      if (tc_enabled && plan_ok[op]) {
        e = conv3_forward_tc(plans[op], out_f32, skip, tc_err, s);
      } else
        e = conv3_forward(conv_desc(*this, op, out_f32, skip), s);
    } else {
      const UnetUpSpec& u = kUnetUp[-1 - op];
      const int lc = kUnetTensor[u.in].level, lf = kUnetTensor[u.out].level;
      e = upsample_forward(dims[lc], dims[lf], kUnetTensor[u.out].ch, act[u.in], act[u.skip], act[u.out], skip, s);
    }
    launches++;
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t UnetNet::backward(cudaStream_t s) {
  cudaError_t e = cudaSuccess;
  for (int t = 1; t < kUnetTensors - 1 && e == cudaSuccess; t++)
    e = cudaMemsetAsync(grad[t], 0, (size_t)nvox[kUnetTensor[t].level] * kUnetTensor[t].ch * sizeof(float), s);
  for (int i = kUnetConvs + 1; i >= 0 && e == cudaSuccess; i--) {
    const int op = kOrder[i];
    if (op >= 0) {
      const UnetConvSpec& c = kUnetConv[op];
      ConvDesc d = conv_desc(*this, op, out);
      float* g = grad[c.out];
      if (c.act) {
        e = act_backward(nvox[kUnetTensor[c.out].level] * kUnetTensor[c.out].ch, act[c.out], g, s);
        launches++;
        if (e != cudaSuccess) break;
      }
      if (c.in != 0) {
        e = conv3_dgrad(d, g, grad[c.in], 1, nullptr, 0, s);
        launches++;
        if (e != cudaSuccess) break;
      }
      e = conv3_wgrad(d, g, G + unet_weight_offset(op), G + unet_bias_offset(op), s);
      launches += 2;
    } else {
      const UnetUpSpec& u = kUnetUp[-1 - op];
      const int lc = kUnetTensor[u.in].level, lf = kUnetTensor[u.out].level;
      const int ch = kUnetTensor[u.out].ch;
      e = upsample_backward(dims[lc], dims[lf], ch, grad[u.out], grad[u.in], s);
      if (e == cudaSuccess) e = add_f32(nvox[lf] * ch, grad[u.out], grad[u.skip], s);
      launches += 2;
    }
  }
  return e;
}

cudaError_t UnetNet::adam(cudaStream_t s, float lr, float gscale) {
  adam_t++;
  packs_dirty = true;
  launches++;
  return adam_step(nparam, P, G, M1, M2, Pb, lr, 0.9f, 0.999f, 1e-8f, adam_t, gscale, s);
}

}  // namespace cfd
