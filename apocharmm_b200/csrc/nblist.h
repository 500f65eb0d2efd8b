// Tiled neighbour list: column sort into 32-atom clusters, warp-ballot tile
// search over cluster bounding boxes, per-tile 32x32 exclusion bitmasks.
//
// Replaces the reference's CudaNeighborList<32> (sort: src/CudaNeighborListSort.cu,
// build: src/CudaNeighborListBuild.cu:337-1700).  Differences by design:
//  * no host round trips: every size lives in device memory, so a rebuild
//    can sit inside a CUDA graph;
//  * the atom order inside a column is fully determined by (z, atom index),
//    so the sorted order, the tile list and the masks are deterministic;
//  * a tile carries its own periodic image code and, only when one of its
//    pairs is a topological 1-2/1-3/1-4 exclusion, the index of its mask (32
//    words, bit j of word i set = pair (i, j) excluded) in a compact mask
//    array; padding slots and the lower triangle of a cluster's tile with
//    itself are skipped by the kernels, so most tiles need no mask.
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "common.h"

namespace apo {

// One system of the list: its own box, list radius and x-y columns.  Several
// independent systems share one list (one set of kernels per rebuild):
// their columns are numbered consecutively, so clusters, tiles and work
// items never mix systems and every work item carries its system index.
struct NbSysDims {
  float Lx = 0, Ly = 0, Lz = 0;      // box
  float rlist = 0;                   // list radius (cutnb)
  double Lxd = 0, Lyd = 0, Lzd = 0;  // box, full precision
  int ncx = 1, ncy = 1;              // cell columns in x, y
  int col_off = 0;                   // first global column
  int atom_off = 0, natom = 0;       // global atom range
  int pad = 0;
};

struct NbListDims {
  int natom = 0;                  // all systems
  int nsys = 1;
  int ncol = 0;                   // all systems
  int slot_cap = 0;               // padded sorted slots
  int tile_cap = 0, work_cap = 0;
  int mask_cap = 0;               // tiles with an exclusion mask
  int tiles_per_work = 8;
  int sort_cap = 4096;            // max atoms in one column
};

// A tile's image code and mask index, packed in its second int.
__host__ __device__ inline int tile_image(int packed) { return packed & 31; }
__host__ __device__ inline int tile_mask(int packed) { return (packed >> 5) - 1; }  // -1: none
// the pairs a cluster's tile with itself skips: j <= i, as a mask word of lane i
__host__ __device__ inline unsigned self_tile_word(int i) {
  return i == 31 ? 0xffffffffu : ((2u << i) - 1u);
}

struct NbListSystem {
  int natom;
  double Lx, Ly, Lz;
  float rlist;
};

class NeighborList {
 public:
  NeighborList() = default;
  ~NeighborList();
  NeighborList(const NeighborList &) = delete;
  NeighborList &operator=(const NeighborList &) = delete;

  // topology-dependent set-up of one system
  void setup(int natom, double Lx, double Ly, double Lz, float rlist,
             const std::vector<int> &excl_ptr, const std::vector<int> &excl_idx,
             const int *d_vdwtype, int tiles_per_work = 8);
  // several systems, atoms concatenated in order; exclusion CSR and LJ types
  // in global atom numbering
  void setup(const std::vector<NbListSystem> &systems, const std::vector<int> &excl_ptr,
             const std::vector<int> &excl_idx, const int *d_vdwtype, int tiles_per_work = 8);
  void set_tiles_per_work(int tpw);
  // full rebuild from global-order coordinates (device float4 x,y,z,q)
  void build(const float4 *d_xyzq, cudaStream_t s);
  // refresh the sorted, cluster-local coordinates from the FP64 state
  void refresh(cudaStream_t s);
  // FP64 state coordinates (atom order, x y z q) the sorted single-precision
  // coordinates are formed from
  void set_state_coordinates(const double4 *c) { m_coords = c; }
  // grow capacities if the last build used more than `fill` of them (sync)
  bool ensure_capacity(const float4 *d_xyzq, cudaStream_t s, double fill = 0.8);
  // tile and work-item capacity set by hand (the buffers are reallocated)
  void set_capacity(int tile_cap, int work_cap);
  void clear_error(cudaStream_t s);
  // a new box for system `sys` with the same columns (a box that changes
  // every step under pressure control); the next build uses it.  The
  // caller has synchronised the stream the list's kernels run on.
  void set_box(int sys, double Lx, double Ly, double Lz);
  // keep the built list under a new box: every slot's periodic shift k L
  // moves with the box (k kept), so the list stays valid between builds
  // while the box changes a little every step; the old and new edges are
  // in device memory (3 doubles each; nothing happens once `err` is set)
  // and the device dims are left alone
  void rescale_box_device(const double *old_box, const double *new_box, const unsigned *err,
                          cudaStream_t s);
  // the host copy of a box the device dims already hold
  void set_box_host(int sys, double Lx, double Ly, double Lz);
  NbSysDims *device_dims() { return m_sys; }

  const NbListDims &dims() const { return m_d; }
  const std::vector<NbSysDims> &system_dims() const { return m_sys_h; }
  int num_columns() const { return m_d.ncol; }
  // device arrays
  int *perm = nullptr;          // slot -> atom (-1 = padding)
  int *glo2loc = nullptr;       // atom -> slot
  float4 *slot_shift = nullptr; // image shift added to the atom's coordinates
  // Sorted coordinates are stored relative to an origin per 32-atom cluster
  // (a multiple of 1/64 A, exact in single precision): xyzq_s = FP64 state
  // + slot_off, rounded once; the absolute wrapped position is xyzq_s +
  // cl_origin[slot / 32].  Pair differences then carry the rounding of
  // coordinates a few A from the origin instead of up to half a box.
  double4 *slot_off = nullptr;  // image shift - cluster origin, FP64
  float4 *cl_origin = nullptr;  // per cluster
  float4 *xyzq_s = nullptr;     // sorted, cluster-local coordinates + charge
  int *type_s = nullptr;        // sorted LJ type
  int2 *tiles = nullptr;        // (j cluster, image code | (mask index + 1) << 5)
  unsigned *masks = nullptr;    // 32 words per masked tile
  int4 *work = nullptr;         // (i cluster, first tile, end tile, system)
  int *counts = nullptr;        // [0] slots, [1] tiles, [2] work items, [3..4] scan
                                // carries, [5] masked tiles, [6..7] direct-space
                                // schedule counters
  unsigned *error = nullptr;    // DeviceError bits
  int *cl_sys = nullptr;        // cluster -> system
  int *sys_of_atom = nullptr;   // atom -> system

  // host copies of the counts (valid after sync_counts)
  int h_counts[3] = {0, 0, 0};
  void sync_counts(cudaStream_t s);
  unsigned read_error(cudaStream_t s);

 private:
  void alloc();
  void release();
  NbListDims m_d;
  std::vector<NbSysDims> m_sys_h;
  NbSysDims *m_sys = nullptr;   // device copy
  int *m_col_sys = nullptr;     // column -> system
  const int *m_vdwtype = nullptr;
  const double4 *m_coords = nullptr;
  int *m_excl_ptr = nullptr, *m_excl_idx = nullptr;
  int *m_col_count = nullptr, *m_col_start = nullptr;
  int *m_atom_col = nullptr, *m_atom_rank = nullptr;
  float4 *m_atom_shift = nullptr;
  float *m_tmp_key = nullptr, *m_atom_z = nullptr;
  int *m_tmp_idx = nullptr;
  int *m_cl_col = nullptr;
  float4 *m_bb_c = nullptr, *m_bb_h = nullptr;
  int *m_tile_count = nullptr, *m_tile_start = nullptr, *m_work_start = nullptr;
};

}  // namespace apo
