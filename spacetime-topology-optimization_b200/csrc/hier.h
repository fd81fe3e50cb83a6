// Host-side description of a device multigrid hierarchy (the object behind stt_hier*).
//
// All device arrays live in one caller-owned workspace, carved by plan_hierarchy().
// Level 0 keeps the (copied) element densities and the lumped reaction diagonal;
// every coarser level keeps its Galerkin operator as a symmetric 9-point block
// stencil: per node the centre block and the E, S, SE, SW coupling blocks (the other
// four couplings are the transposes of the neighbours' blocks), each D x D, stored
// coefficient-major ([row][coef][node]) so a warp reads one coefficient coalesced.
// The coarsest level is factorised by a block-banded FP64 Cholesky.
#pragma once

#include <atomic>
#include <mutex>

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "../../include/sttb200.h"

namespace stt {

constexpr int kMaxLevels = 24;

inline int stencil_coefs(int d) { return 5 * d * d; }

struct LevelDesc {
  int nelx, nely;  // elements of this level
  int kx, ky;      // coarsening factors to the next level (1, 1 at the coarsest)
  int nnx, nny;
  long long nnode, ndof, nel;
  long long rs_rho;  // row stride of rho64 / rho32: nel rounded up to 4 (16-byte aligned rows)
  uint8_t* fixed;  // [nnode] bit i = dof i fixed
  // level 0 only
  double* rho64;    // [hrows][nel]
  float* rho32;     // [hrows][nel] (FP32 precision only)
  double* rdiag64;  // [hrows][ndof] lumped reaction diagonal, or null
  float* rdiag32;
  // levels >= 1 (and level 0 when it is also the coarsest)
  double* st64;  // [hrows][NS][nnode]
  float* st32;   // [hrows][NS][nnode] (FP32 precision only)
};

struct CoarseDesc {
  int n;             // dofs of the coarsest level
  int B;             // block size (>= half bandwidth)
  int nb;            // blocks, n padded to nb * B
  int by_col;        // dof ordering: 1 = column-major nodes (nny < nnx), 0 = row-major
  double* blocks;    // [hrows][nb][4][B][B]: Dinv, Dinv^T, E, E^T (E_k = L_{k,k-1})
  double* inv;       // [hrows][nb B][nb B] explicit inverse (FP32 cycles, B <= 64), or null
};

// The coarsest level's factorisation runs on a stream of its own, concurrently with the
// caller's next work (a solve's initialisation and first descent); `ready` marks its end.
// Shared by a hierarchy and its row-selected views; the last one destroyed waits for it.
struct CoarseSync {
  int device = 0;
  cudaStream_t side = nullptr;
  cudaEvent_t built = nullptr, ready = nullptr;
  cudaEvent_t factored = nullptr;  // the band factor is done (the inverse may still run)
  std::atomic<int> refs{1};
  // an FP32 hierarchy's first coarse solve takes the block solves, which need only the
  // factor, so it does not wait for the explicit inverse (set at the build, taken once)
  std::atomic<int> first_cycle{0};
  // level 1's FP64 stencil not yet assembled (an FP32 hierarchy swept from the densities
  // builds only the FP32 diagonal its cycle reads); the first entry point that reads the
  // FP64 stencil assembles it, under l1_mu.  Shared by the hierarchy's views.
  std::atomic<int> l1_pending{0};
  std::mutex l1_mu;
};

struct stt_hier_impl {
  int d, nelx, nely, hrows, precision, nlevels, mce;
  LevelDesc lv[kMaxLevels];
  CoarseDesc co;
  double KE[64];
  int modal;         // KE has the modal form (march_modal); mq holds its constants
  double mq[8];
  int l1;            // level 1 is applied from the level-0 densities (l1_sweep_kernel)
  double l1m[9][21]; // per child m of a level-1 element: T G_m T^T / 16, packed upper triangle
  int l1par;         // 2 x 2 children whose M_m are mirror images of M_0 (l1_mirror_classes)
  double* tables;    // device: per transition S[9][64], G[9][64], GM[9][64]
  double* gtables;   // device: level-0 grandchildren of a level-2 element, H[81][64], HM[81][64]
  double* keffA;     // build temporaries: element matrices of levels 3, 5, ...
  double* keffB;     // ... and of levels 2, 4, ...
  const int* row_map;  // batch row -> hierarchy row (device), or null
  int has_reaction;    // level 0 carries a lumped reaction (drain) term
  int* status;         // device status word of the build (bit 0: pivot <= 0, bit 1: band)
  CoarseSync* sync;    // the coarse factorisation's stream and completion event
  long long ws_bytes;
  int tune_pcg_band = 0;  // launch tuning of the solves on this hierarchy (stt_hier_tune; 0: heuristics)
  int tune_waves = 0;
};

inline int level_node_count(int nelx, int nely) { return (nelx + 1) * (nely + 1); }

// Plans level shapes and carves the workspace (base may be null to only size it).
// Returns the bytes needed.
long long plan_hierarchy(stt_hier_impl& h, char* base);

// The build's device status word (copied to the host) as an STT error code.
int hier_status_code(int s);
// Assembles level 1's deferred FP64 stencil (see CoarseSync::l1_pending) before a read of it.
int ensure_level1_fp64(const stt_hier* h, int level, cudaStream_t st);

}  // namespace stt

struct stt_hier : stt::stt_hier_impl {};
