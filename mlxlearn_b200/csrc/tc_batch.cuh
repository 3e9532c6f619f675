// Work description shared by the tcgen05 screen and the batched planner.
//
// A screen launch walks work units: (problem, query tile of 128 rows, range
// of 256-row reference tiles).  A single kneighbors call is one problem whose
// units are dealt round-robin; a batched launch reads a host-built unit list
// whose per-CTA ranges were balanced on the host (batch.cu).
#pragma once
#include "internal.cuh"
#include "sinks.cuh"

namespace b2k {

// Problems of one batched launch share at most this many operand groups; a
// group is a set of problems with the same padded width dp, whose bf16
// operands live in one concatenated buffer addressed by one tensor map.
constexpr int kBatchGroups = 4;

struct TcProblem {
  int m;                // query rows
  int KB;               // 64-column blocks of the padded width
  int n_tiles;          // 256-row reference tiles
  int tiles_per_split;  // reference tiles per split (list slot = first tile / this)
  int exclude_self;
  int group;            // operand group (tensor maps) of the launch
  int a_row0;           // first row of the problem's queries in the group's A buffer
  int b_row0;           // first row of the problem's reference rows in the group's B buffer
  long long q_offset;
  const float* E;       // [m_pad] screen error bound per query row
  const int* perm;      // tile row -> original query row (or null)
  const int* self_col;  // training row -> its reference column (grouped operand), or null
  const int* nxu;       // u8 screen: ||x||^2 per reference row (exact), else null
  SinkArgs sink;
};

// One batched screen launch.  `items` are int4 (problem, query tile, first
// reference tile, end reference tile); CTA b runs items [cta_begin[b],
// cta_begin[b+1]).
struct TcBatchLaunch {
  CUtensorMap a[kBatchGroups], b[kBatchGroups], baug[kBatchGroups];
  CUtensorMap aaug;
  int groups;
  const TcProblem* probs;
  const int4* items;
  const int* cta_begin;
  int* item_counter;  // claimed in order from `items` when set (then cta_begin is unused)
  int n_items;
  int grid;
  int KB_max;
  int kmax;       // heap width class: 8, 12, 16, or 64 (lazy tracker, k > 16)
  int ew;         // epilogue warps: 4, 8, or 16 (heap widths <= 16)
  bool a_stream;  // stream the query tile with every block (KB_max > 4)
  int* status;
};

// Validates the (kmax, ew) pair and sets the kernel's shared-memory limit
// (call before stream capture).  Returns 0 or a cudaError_t.
int prepare_screen_tc_batch(int kmax, int ew, bool a_stream, int KB_max);
int launch_screen_tc_batch(const TcBatchLaunch& L, cudaStream_t st);

}  // namespace b2k
