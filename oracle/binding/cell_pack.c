/*
 * The two functions a Disco2 maintainer adds to src/Cell/ to hand the cell
 * state to the B200 library and take it back (compiled with the reference's
 * own headers).  The reference keeps the cells of a rank as one contiguous
 * block theCells[0][0] in (k, i, j) order (cell_create,
 * src/Cell/cell_create_destroy.c:23-95); the library's dgpu_set_state /
 * dgpu_get_state take the same order as NUM_Q-wide prim rows plus the phi
 * edge tiph and width dphi of every cell.
 */
#define CELL_PRIVATE_DEFS
#include "Headers/Cell.h"
#include "Headers/Sim.h"
#include "Headers/header.h"

#include "cell_pack.h"

int cell_pack_count(struct Sim *s) {
  int i, n = 0;
  for (i = 0; i < sim_N(s, R_DIR); ++i) n += sim_N_p(s, i) * sim_N(s, Z_DIR);
  return n;
}

void cell_pack(struct Cell ***c, struct Sim *s, double *prim, double *tiph, double *dphi) {
  int n, q, N = cell_pack_count(s), NQ = sim_NUM_Q(s);
  struct Cell *b = c[0][0];
  for (n = 0; n < N; ++n) {
    for (q = 0; q < NQ; ++q) prim[(long)n * NQ + q] = b[n].prim[q];
    tiph[n] = b[n].tiph;
    dphi[n] = b[n].dphi;
  }
}

void cell_unpack(struct Cell ***c, struct Sim *s, const double *prim, const double *cons, const double *tiph,
                 const double *dphi) {
  int n, q, N = cell_pack_count(s), NQ = sim_NUM_Q(s);
  struct Cell *b = c[0][0];
  for (n = 0; n < N; ++n) {
    for (q = 0; q < NQ; ++q) {
      b[n].prim[q] = prim[(long)n * NQ + q];
      b[n].cons[q] = cons[(long)n * NQ + q];
    }
    b[n].tiph = tiph[n];
    b[n].dphi = dphi[n];
  }
}
