// Shared declarations of the learned preconditioner (mac_unet.cu, mac_unet_host.cu).
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace mac {
namespace unet {

struct LayerDef {
  int cin, cout, taps, relu, real_cin, real_cout;
};
constexpr int kNumLayers = 13;
extern const LayerDef kLayers[kNumLayers];

// Activation (and matching gradient) tensors.
enum Act { IN0, A1, S1, P1, A2, S2, P2, A3, B3, U2, C2, D2, U1, C1, D1, GOUT, GUP2, GUP1, kNumAct };
extern const int kActCh[kNumAct];
extern const int kActLvl[kNumAct];

// One gathered source of a convolution: c channels, stored at full (shift 0)
// or half (shift 1) resolution of the convolution's grid.
struct Src {
  const __nv_bfloat16* p;
  int c, shift;
};

struct ConvArgs {
  Src s1, s2;                  // K channels = s1.c + s2.c
  const __nv_bfloat16* gate;   // input gradient: gathered values times (gate > 0)
  const __nv_bfloat16* wt;     // weights [taps][cout][cin]
  const float* bias;           // forward only
  __nv_bfloat16* d1;           // output channels [0, c1)
  int c1;
  __nv_bfloat16* d2;           // output channels [c1, N)
  float* f32;                  // forward output layer: channel 0 in FP32
  int taps, relu;
  int n, d, h, w;              // grid of the output (and of the gather)
  int* err;
};

struct WgradArgs {
  Src s1, s2;                  // the layer's forward input
  const __nv_bfloat16* g;      // gradient at the layer's output
  const __nv_bfloat16* gate;   // the layer's output (ReLU) or null
  float* dw;                   // [taps][cout][cin], accumulated
  int taps;
  int n, d, h, w;
  int vox_per_cta;
  int* err;
};

struct Net;
void destroy(Net* t);
// Buffers of n samples on a d x h x w grid (multiples of 4): residual r and
// mask m to fill, correction z written by apply().
int stage(Net* t, int n, int d, int h, int w, float** r, int8_t** m, float** z);
int apply(Net* t, cudaStream_t st);

}  // namespace unet
}  // namespace mac
