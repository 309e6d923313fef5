// pt_launch.h - launch records shared by the host runtime and the NVRTC-compiled kernels.
#pragma once

#define SNELLY_BLOCK 128  // threads per block of the per-pixel kernels
// Resident blocks per SM the register allocation of the path-per-thread kernel and of the
// wavefront shade stage is held to (65536 registers / (blocks x 128 threads) per thread).
#ifndef SNELLY_MEGA_MIN_BLOCKS
#define SNELLY_MEGA_MIN_BLOCKS 5
#endif
#ifndef SNELLY_SHADE_MIN_BLOCKS
#define SNELLY_SHADE_MIN_BLOCKS 5
#endif

// Render modes (the values of SNELLY_MODE_* in snelly.h).
#define JOB_MODE_PT 0
#define JOB_MODE_NORMALS 1
#define JOB_MODE_AO 2
#define JOB_MODE_PICK 3
#define JOB_MODE_PTSIMPLE 4

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
  int pick_at;           // pick mode: trace the single pixel coordinate (pick_x, pick_y)
  float pick_x, pick_y;  // (gl_FragCoord units of a frame of params.resolution)
} JobRec;

// Wavefront path state and queues of one job (device pointers). Layout shared with the host
// (wavefront.cpp). A path's state is one contiguous record of `rec_f4` float4 slots (the slot
// map is in pt_wavefront.cuh), so that a stage reading it touches a few whole 32-byte sectors
// wherever the path sits in the queue it came from.
#define WF_A 0      // active-path queue counts [2] (ping-pong by iteration parity)
#define WF_S 2      // shadow-ray queue counts [2]
#define WF_C 4      // parked-ray queue counts [2]
#define WF_LEFT 6   // paths with samples of the launch sequence left to finish
#define WF_Q 8      // shade-queue segment counts [2][4]
#define WF_SSS 16   // subsurface-walk queue count (filled by the shade stage, read by the walk stage)
#define WF_WHEAD 17 // the persistent walker's work head over that queue
#define WF_XQ 18    // walks that ended (exit queue count, read by the walk-exit stage)
#define WF_HEAD 19  // extend work heads [2] (ping-pong by iteration parity)
#define WF_VOL 21   // medium-scatter queue count (filled by the shade stage, read by the volume stage)
#define WF_COUNTERS (WF_VOL + 1)
typedef struct WfBuffers {
  float4* rec;      // path records, rec_f4 float4 slots per path
  float4* mt;       // march state of a parked ray (distance, sign, step count), by ray id
  unsigned char* shadow;  // occlusion result per shadow ray (2 per path)
  int* pend;        // rays each path waits for
  int* qa[2];       // active-path queues (continuation rays)
  int* qs[2];       // shadow-ray queues (path * 2 + light)
  int* qc[2];       // parked-ray queues (ray ids: 2 * path + light, or 2 * paths + path)
  int* qshade[2];   // shade queues [2] (ping-pong by iteration parity), 4 segments of `paths`
                    // entries each: finish/miss, surface, metal, dielectric
  int* qsss;        // paths whose surface vertex chose the subsurface walk (one iteration's)
  int* qexit;       // paths whose walk the persistent walker finished (one iteration's)
  int* qvol;        // paths whose vertex scatters in the heterogeneous medium (one iteration's)
  int* cnt;         // counters (WF_*)
  int paths;
  int pixel_begin;  // contiguous range (pixel_group 0): its first pixel; interleaved: the range's index
  int pixel_group;  // > 0: the image's groups of pixel_group pixels are dealt to the ranges in turn
  int pixel_parts;  // ranges the groups are dealt to
  int rec_f4;       // float4 slots per path record (checked against the module's layout)
  int slot;         // the job's constant-memory parameter and uniform slot
  int samples;      // samples per pixel one generate launch starts: a path that finishes its
                    // pixel's sample starts the pixel's next one in place until this many are done
  int vol_stage;    // 1: the shade stage hands medium collisions to the volume stage (queue qvol)
} WfBuffers;
