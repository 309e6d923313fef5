// pt_launch.h - launch records shared by the host runtime and the NVRTC-compiled kernels.
#pragma once

#define SNELLY_BLOCK 128  // threads per block of the per-pixel kernels

// One job's slice of a batched launch. Pointers are device addresses of the job's SoA buffers.
typedef struct JobRec {
  uint4* rng;            // 4 LCG lanes per pixel
  float4* acc;           // Kahan sums (X, Y, Z) and frame count (w)
  float4* comp;          // Kahan compensations
  double* acc64;         // optional FP64 sums, 4 per pixel (or null)
  float4* out;           // resolve target: mean XYZ and count
  unsigned long long seed;
  int width, height;
  int pixel_begin;       // first pixel index covered by this launch
  int pixel_count;       // pixels covered by this launch
  int slot;              // index into the module's constant-memory parameter banks
  int mode;              // SNELLY_MODE_*
} JobRec;
