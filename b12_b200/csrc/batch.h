// Batched box-image kernels shared by the batch (batch.cu) and the job server (serve.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.h"

namespace b12g {

constexpr uint32_t kMaxInstances = 4096;

struct Tuning {
  uint32_t threads = 256;
  uint32_t ppt = 1;                 // test points per thread
  uint32_t chunk = 8192;            // points per work-queue item
};

// ------------------------------------------------------------------------ device side
struct BatchArgs {
  Domain dom;
  MapParams map;                    // h, steps, table; p[] per instance from `params`
  GridParams grid;
  uint64_t points;                  // per box
  const double* params;             // instance x 6
  const uint8_t* depths;            // instance -> target depth (row kernel)
  uint32_t n_inst;                  // instances in this launch (active prefix)
  const uint32_t* off;              // n_inst + 1 parent offsets
  const uint64_t* codes;            // parents
  int depth;                        // depth of the children (subdivision step)
  const uint8_t* inst_depth;        // per-instance children depth (nullptr: `depth` for all)
  DepthConst dc;                    // constants of `depth` when every instance has it
                                    // (launch_batch_image fills them in)
  LeafHash hash;
  uint8_t* hit;
  uint32_t hit_cap;
  uint32_t* queue;                  // work-queue head (zeroed before the launch)
  uint32_t chunk;
  uint32_t* error;
  // optional: every point's target (global child index, kInvalidIndex when its box is
  // not a child of a leaf, kOutsideIndex when it left the domain) for the instances with
  // tgt_base[i] != ~0: targets[tgt_base[i] + (child - 2 off[i]) * points + k]
  uint32_t* targets;
  const uint64_t* tgt_base;
};

// transition rows of the instances finishing in a step, from the targets their last
// step stored and the ranks of that step's compaction (no map evaluation)
struct TargetRowArgs {
  uint32_t n_inst;                  // finishing instances
  const uint32_t* child_off;        // n_inst + 1: prefix of their children counts
  const uint32_t* child_base;       // n_inst: global index of each one's first child
  const uint32_t* row_off;          // n_inst: each one's first row (arena position)
  const uint32_t* rank;             // the step's compaction ranks (children + 1 entries)
  const uint32_t* targets;          // child_off[n_inst] x points
  const uint64_t* arena;            // final leaves (for the single-leaf rule)
  uint32_t points;
  int keep_lost;
  uint32_t* stage_col;
  uint32_t* stage_cnt;
  uint32_t* row_count;
};

// transition rows of the finished leaves of all instances: warp per row, targets found
// by (instance, code); column = target index within its instance
struct BatchRowArgs {
  Domain dom;
  MapParams map;
  GridParams grid;
  uint64_t points;
  const double* params;
  const uint8_t* depths;
  uint32_t n_inst;
  const uint32_t* off;            // arena-order region offsets (n_inst + 1)
  const uint32_t* inst_of;        // arena index -> sorted position (params, depth)
  const uint64_t* codes;          // final arena
  LeafHash hash;
  int keep_lost;
  uint32_t* stage_col;
  uint32_t* stage_cnt;
  uint32_t* row_count;
};

// the image kernel's launch shape for a map family: the autotuned one when a batch of
// this process has tuned it on `device`, else the shape the tuner settles on for it
Tuning batch_tuning(int device, uint32_t map_kind, uint32_t arith, uint32_t grid_kind, uint32_t dim);

// launches (batch.cu)
bool batch_supported(uint32_t map_kind, uint32_t arith, uint32_t grid_kind);
cudaError_t launch_batch_image(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, const Tuning& tu,
                               const BatchArgs& a, cudaStream_t s);
cudaError_t launch_batch_rows(uint32_t map_kind, uint32_t arith, uint32_t grid_kind, const BatchRowArgs& a,
                              uint32_t max_rows, cudaStream_t s);
// lookup table over (instance, code) of n_inst concatenated code segments
cudaError_t launch_batch_hash(const uint64_t* codes, const uint32_t* off, uint32_t n_inst, LeafHash h,
                              uint32_t code_cap, uint32_t* error, cudaStream_t s);
cudaError_t launch_target_rows(const TargetRowArgs& a, uint32_t max_children, cudaStream_t s);
// survivors per instance from the hit mask of the instances' (implicit) children
cudaError_t launch_inst_count(const uint8_t* hit, const uint32_t* off, uint32_t n_inst, uint32_t* cnt,
                              uint64_t hit_cap, uint32_t* error, cudaStream_t s);

}  // namespace b12g
