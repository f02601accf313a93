// Internal interface of the projection / CG stage (see sw_project.cu).
#pragma once

#include "sw_common.cuh"

namespace sw {

// Element strides of an input field: element (x, y, z) at x*sx + y*sy + z*sz.
struct InStride {
  long long sx, sy, sz;
};

// Scalar state of one CG solve, advanced on the device by the last block of
// each launch.
struct CgState {
  double rs;      // r.r of the current residual (rs_old)
  double rs0;     // max(r0.r0, eps64)
  double alpha, beta;
  double rel;     // sqrt(rs_new / rs0) of the last update
  double maxdiv;  // max |div_c f| of the masked input
  double tol;
  int iters;      // completed x updates
  int reason;     // enum sw_cg_reason
  int k;          // index of the next apply (selects the p buffer)
  int max_iters;
  unsigned int ticket;
};

static_assert(sizeof(CgState) <= 128, "the grid barrier shares the state's 256-byte slot");

// Grid-wide barrier of the persistent CG kernel (zeroed before each launch):
// arrivals, generation, and an error word set when a wait runs out.
struct CgGrid {
  unsigned int count;
  unsigned int gen;
  int error;
  int pad;
};
// The barrier of a single solve lives 128 bytes after its state.
inline CgGrid* cg_grid_of(CgState* st) { return (CgGrid*)((char*)st + 128); }

// One solve in a launch's instance table.
//   op 0: the projection's Poisson operator A = -div_c(grad_c .)
//         (src/shearwave/solver.py:1024-1026), rhs = -div_c(mask f);
//   op 1: the static elastic operator A = -mu L7(.) (solver.py:596-597),
//         rhs = mask b; no non-finite breaks and no early exit, like the
//         reference's elastic_solve_static loop (solver.py:605-623).
struct CgInst {
  Geom g;
  TileSpace ts;
  double c2x, c2y, c2z;  // 1 / (2 h)
  double ihx2, ihy2, ihz2;  // 1 / h^2 (op 1)
  double *x, *r, *p0, *p1, *ap;
  double* muf;           // mu on interior cells, FP64 (op 1)
  double mu_s;           // scalar mu when no field is given (op 1)
  double2* partials;     // per tile: (sum, max)
  CgState* st;
  int tile_base;         // first global tile index of this instance
  int op;
};

size_t align_up(size_t v, size_t a);
TileSpace cg_tiles(const Geom& g);
size_t cg_workspace_bytes(const Geom& g, const TileSpace& ts);

// Project one 3-component field (any dtype / strides) into `out`
// (3 padded FP64 components).  Synchronises `s`.
int project_field(int dtype, const void* fx, const void* fy, const void* fz, InStride fs,
                  const Geom& g, double dX, double dY, double dZ, double tol, int max_iters,
                  double* out, void* ws, size_t ws_bytes, sw_cg_stats* stats, cudaStream_t s);

}  // namespace sw
