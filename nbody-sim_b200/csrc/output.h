// output.h -- the GPU output pipeline of an engine (output.cu).
#pragma once
#include <cuda_runtime.h>

#include "../../include/nbody_b200.h"
#include "kernels.cuh"

namespace nb {

struct OutputPipe {
  struct Slot {
    float* snap[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};  // x..vz, device
    nbody_aggregate* drec = nullptr;
    int* dcount = nullptr;
    float* hx = nullptr;              // pinned: x, y, z
    uint16_t* hagg = nullptr;         // pinned: agg_size
    nbody_aggregate* hrec = nullptr;  // pinned: records
    int* hcount = nullptr;            // pinned: record count
    int* hstatus = nullptr;           // pinned: device status of this frame
    cudaEvent_t snap_ready = nullptr, done = nullptr;
    bool pending = false;
    float time = 0.f;
    int frame = 0;
    unsigned long long seq = 0;
  };

  int n = 0, leaf_max = 8, next = 0;
  unsigned long long seq = 0;
  cudaStream_t os = nullptr;
  TreeWork tw;
  int *parent = nullptr, *labels = nullptr, *sizes = nullptr, *ngroups = nullptr;
  uint16_t* agg = nullptr;
  int* spill = nullptr;
  int spill_cap = 4096;
  int* work = nullptr;
  uint32_t *keys = nullptr, *vals = nullptr, *keys_alt = nullptr, *vals_alt = nullptr;
  uint32_t *flag = nullptr, *slotix = nullptr, *scan_tmp = nullptr;
  Slot slot[2];

  OutputPipe(int n, int leaf_max);
  ~OutputPipe();
  // Slot for the next frame (throws when both are in flight); the caller
  // writes the snapshot into slot[k].snap on its engine stream, then launch().
  int begin_slot();
  void launch(int k, cudaStream_t engine, float link_length, float particle_mass,
              float sim_time, int frame_index);
  // Oldest frame in flight: waits for it and points out at its pinned buffers.
  void wait(nbody_frame* out);

 private:
  void enqueue(Slot& sl, float link_length, float particle_mass);
};

}  // namespace nb
