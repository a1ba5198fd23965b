/*
 * Checkpoint and restart in the reference's layout (src/IO/io_hdf5.c,
 * src/IO/io_buffer.c, the restart branch of src/main.c:95-117), through the
 * library-free HDF5 subset of dgpu_h5.c.  Host code.
 *
 * A checkpoint holds T [1] = t, GravMass [2][4] = (r, phi, M, omega) of each
 * mass, and Data [Ncells][NUM_Q+3]: per cell, in (k, i, j) order with the
 * ghost annuli and layers, tiph, the annulus centre 0.5*(FacePos(i-1) +
 * FacePos(i)), the layer centre 0.5*(FacePos(k-1, Z) + FacePos(k, Z)) and the
 * NUM_Q primitives (io_setbuf, src/IO/io_buffer.c:26-58).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dgpu_ctx.h"
#include "dgpu_h5.h"

#define fail dctx_fail

static int arg_ok_path(const char *path) { return path && path[0]; }

int dgpu_hdf5_out(const char *path, double t, const double *gravmass, const double *data, long long nrows, int ncols) {
  h5_dataset ds[3];
  char err[384];
  if (!arg_ok_path(path) || !gravmass || nrows < 0 || ncols < 1 || (nrows > 0 && !data))
    return fail(NULL, DGPU_ERR_ARG, "bad arguments to dgpu_hdf5_out");
  ds[0].name = "T";
  ds[0].rank = 1;
  ds[0].dims[0] = 1;
  ds[0].dims[1] = 0;
  ds[0].data = &t;
  ds[1].name = "GravMass";
  ds[1].rank = 2;
  ds[1].dims[0] = 2;
  ds[1].dims[1] = 4;
  ds[1].data = gravmass;
  ds[2].name = "Data";
  ds[2].rank = 2;
  ds[2].dims[0] = (uint64_t)nrows;
  ds[2].dims[1] = (uint64_t)ncols;
  ds[2].data = data;
  switch (h5_write(path, ds, 3, err, (int)sizeof(err))) {
    case 0: return DGPU_OK;
    case -2: return fail(NULL, DGPU_ERR_NOMEM, "%s", err);
    default: return fail(NULL, DGPU_ERR_IO, "%s", err);
  }
}

int dgpu_hdf5_dataset(const char *path, const char *name, int *rank, long long *dims, double *data) {
  char err[384];
  int r, rk;
  uint64_t d[H5_MAX_RANK] = {0, 0};
  if (!arg_ok_path(path) || !name || !rank || !dims) return fail(NULL, DGPU_ERR_ARG, "bad arguments to dgpu_hdf5_dataset");
  if (h5_read(path, name, &rk, d, NULL, 0, 0, err, (int)sizeof(err))) return fail(NULL, DGPU_ERR_IO, "%s", err);
  if (data && h5_read(path, name, &rk, d, data, 0, rk ? d[0] : 1, err, (int)sizeof(err)))
    return fail(NULL, DGPU_ERR_IO, "%s", err);
  *rank = rk;
  for (r = 0; r < H5_MAX_RANK; ++r) dims[r] = r < rk ? (long long)d[r] : 1;
  return DGPU_OK;
}

int dgpu_hdf5_dims(const char *path, long long *nrows, int *ncols) {
  char err[384];
  int rank;
  uint64_t dims[H5_MAX_RANK] = {0, 0};
  if (!arg_ok_path(path) || !nrows || !ncols) return fail(NULL, DGPU_ERR_ARG, "bad arguments to dgpu_hdf5_dims");
  if (h5_read(path, "Data", &rank, dims, NULL, 0, 0, err, (int)sizeof(err))) return fail(NULL, DGPU_ERR_IO, "%s", err);
  if (rank != 2) return fail(NULL, DGPU_ERR_IO, "%s: Data has rank %d, not 2", path, rank);
  *nrows = (long long)dims[0];
  *ncols = (int)dims[1];
  return DGPU_OK;
}

int dgpu_hdf5_in(const char *path, long long row0, long long nrows, int ncols, double *t, double *gravmass,
                 double *data) {
  char err[384];
  int rank;
  uint64_t dims[H5_MAX_RANK] = {0, 0};
  double tt;
  if (!arg_ok_path(path) || row0 < 0 || nrows < 0 || ncols < 1 || (nrows > 0 && !data))
    return fail(NULL, DGPU_ERR_ARG, "bad arguments to dgpu_hdf5_in");
  /* T: the reference reads one value through a [1] memory space */
  if (h5_read(path, "T", &rank, dims, NULL, 0, 0, err, (int)sizeof(err))) return fail(NULL, DGPU_ERR_IO, "%s", err);
  if (rank != 1 || dims[0] != 1) return fail(NULL, DGPU_ERR_IO, "%s: T is not a single value", path);
  if (h5_read(path, "T", &rank, dims, &tt, 0, 1, err, (int)sizeof(err))) return fail(NULL, DGPU_ERR_IO, "%s", err);
  if (t) *t = tt;
  if (h5_read(path, "GravMass", &rank, dims, NULL, 0, 0, err, (int)sizeof(err)))
    return fail(NULL, DGPU_ERR_IO, "%s", err);
  if (rank != 2 || dims[0] != 2 || dims[1] != 4) return fail(NULL, DGPU_ERR_IO, "%s: GravMass is not [2][4]", path);
  if (gravmass && h5_read(path, "GravMass", &rank, dims, gravmass, 0, 2, err, (int)sizeof(err)))
    return fail(NULL, DGPU_ERR_IO, "%s", err);
  if (h5_read(path, "Data", &rank, dims, NULL, 0, 0, err, (int)sizeof(err))) return fail(NULL, DGPU_ERR_IO, "%s", err);
  if (rank != 2 || dims[1] != (uint64_t)ncols)
    return fail(NULL, DGPU_ERR_IO, "%s: Data is not [rows][%d] (rank %d, %llu columns)", path, ncols, rank,
                (unsigned long long)dims[1]);
  if ((uint64_t)row0 > dims[0] || (uint64_t)nrows > dims[0] - (uint64_t)row0)
    return fail(NULL, DGPU_ERR_IO, "%s: rows [%lld, %lld) outside Data's %llu rows", path, row0, row0 + nrows,
                (unsigned long long)dims[0]);
  if (nrows > 0 &&
      h5_read(path, "Data", &rank, dims, data, (uint64_t)row0, (uint64_t)nrows, err, (int)sizeof(err)))
    return fail(NULL, DGPU_ERR_IO, "%s", err);
  return DGPU_OK;
}

int dgpu_sim_restart_state(const dgpu_sim *s, const char *path, double *prim, double *tiph, double *dphi,
                           double *gm, double *t) {
  const int NQ = s ? s->NQ : 0, ncols = NQ + 3;
  double *buf, *tp, *dp, gmb[8], tt;
  long idx;
  int q, p, rc;
  if (!s || !arg_ok_path(path)) return fail(NULL, DGPU_ERR_ARG, "bad arguments to dgpu_sim_restart_state");
  buf = (double *)malloc(sizeof(double) * (size_t)ncols * (size_t)s->Ncells);
  tp = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  dp = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  if (!buf || !tp || !dp) {
    free(buf); free(tp); free(dp);
    return fail(NULL, DGPU_ERR_NOMEM, "out of host memory");
  }
  /* cell_create's phi edges and widths, then cell_clean_pi (main.c:74-78):
   * io_readbuf overwrites every tiph, so only dphi = 2pi/N_p survives */
  dsim_initial_tiph(s, tp, dp);
  /* io_hdf5_in + io_readbuf (io_hdf5.c:161-266, io_buffer.c:60-81), one rank:
   * rows [0, Ncells) */
  rc = dgpu_hdf5_in(path, 0, s->Ncells, ncols, &tt, gmb, buf);
  if (rc == DGPU_OK) {
    for (idx = 0; idx < (long)s->Ncells; ++idx) {
      const double *row = buf + (size_t)ncols * (size_t)idx;
      tp[idx] = row[0];
      if (prim) {
        for (q = 0; q < NQ; ++q) prim[(size_t)NQ * (size_t)idx + (size_t)q] = row[3 + q];
        if (s->NumZ == 1) prim[(size_t)NQ * (size_t)idx + 4] = 0.0; /* UZZ */
      }
    }
    /* main.c:111-112: the syncs after the restart; on one rank only the
     * periodic z copy moves data */
    dsim_host_zsync(s, tp, prim);
    if (tiph) memcpy(tiph, tp, sizeof(double) * (size_t)s->Ncells);
    if (dphi) memcpy(dphi, dp, sizeof(double) * (size_t)s->Ncells);
    if (gm) {
      /* gravMass_set_chkpt (GravMass_init.c:86-91) then gravMass_clean_pi
       * (GravMass_misc.c:9-17).  Mdot and Macc are not in the file: the
       * reference leaves them as malloc returned them (gravMass_create,
       * GravMass_create_destroy.c:7-10); they are set to 0 here. */
      for (p = 0; p < 2; ++p) {
        double phi = gmb[4 * p + 1];
        while (phi > 2. * M_PI) phi -= 2. * M_PI;
        while (phi < 0.0) phi += 2. * M_PI;
        gm[6 * p + 0] = gmb[4 * p + 0];
        gm[6 * p + 1] = phi;
        gm[6 * p + 2] = gmb[4 * p + 2];
        gm[6 * p + 3] = gmb[4 * p + 3];
        gm[6 * p + 4] = 0.0;
        gm[6 * p + 5] = 0.0;
      }
    }
    if (t) *t = tt;
  }
  free(buf); free(tp); free(dp);
  return rc;
}

int dgpu_checkpoint_out(dgpu_ctx *c, int inst, const char *path) {
  const struct dgpu_sim *s;
  double *prim, *tiph, *data, gm[12], gmb[8], t, dt;
  long idx = 0;
  int i, j, k, q, p, ncols, rc;
  if (!c) return DGPU_ERR_ARG;
  if (inst < 0 || inst >= c->n_inst || !arg_ok_path(path))
    return fail(c, DGPU_ERR_ARG, "bad arguments to dgpu_checkpoint_out");
  s = c->sims[inst];
  ncols = s->NQ + 3;
  prim = (double *)malloc(sizeof(double) * (size_t)s->NQ * (size_t)s->Ncells);
  tiph = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  data = (double *)malloc(sizeof(double) * (size_t)ncols * (size_t)s->Ncells);
  if (!prim || !tiph || !data) {
    free(prim); free(tiph); free(data);
    return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  }
  rc = dgpu_get_state(c, inst, prim, NULL, tiph, NULL);
  if (rc == DGPU_OK) rc = dgpu_get_gravmass(c, inst, gm);
  if (rc == DGPU_OK) rc = dgpu_get_time(c, inst, &t, &dt);
  if (rc == DGPU_OK) {
    /* io_setbuf (io_buffer.c:26-58) */
    for (k = 0; k < s->NZ; ++k) {
      const double zc = 0.5 * (s->z_faces[k] + s->z_faces[k + 1]);
      for (i = 0; i < s->NR; ++i) {
        const double rc_ = 0.5 * (s->r_faces[i] + s->r_faces[i + 1]);
        for (j = 0; j < s->N_p[i]; ++j, ++idx) {
          double *row = data + (size_t)ncols * (size_t)idx;
          row[0] = tiph[idx];
          row[1] = rc_;
          row[2] = zc;
          for (q = 0; q < s->NQ; ++q) row[3 + q] = prim[(size_t)s->NQ * (size_t)idx + (size_t)q];
        }
      }
    }
    for (p = 0; p < 2; ++p)
      for (q = 0; q < 4; ++q) gmb[4 * p + q] = gm[6 * p + q];
    rc = dgpu_hdf5_out(path, t, gmb, data, s->Ncells, ncols);
    if (rc != DGPU_OK) rc = fail(c, rc, "%s", dgpu_last_error(NULL));
  }
  free(prim); free(tiph); free(data);
  return rc;
}

int dgpu_checkpoint_in(dgpu_ctx *c, int inst, const char *path) {
  const struct dgpu_sim *s;
  double *prim, *tiph, *dphi, gm[12], t;
  int rc;
  if (!c) return DGPU_ERR_ARG;
  if (inst < 0 || inst >= c->n_inst || !arg_ok_path(path))
    return fail(c, DGPU_ERR_ARG, "bad arguments to dgpu_checkpoint_in");
  s = c->sims[inst];
  prim = (double *)malloc(sizeof(double) * (size_t)s->NQ * (size_t)s->Ncells);
  tiph = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  dphi = (double *)malloc(sizeof(double) * (size_t)s->Ncells);
  if (!prim || !tiph || !dphi) {
    free(prim); free(tiph); free(dphi);
    return fail(c, DGPU_ERR_NOMEM, "out of host memory");
  }
  rc = dgpu_sim_restart_state(s, path, prim, tiph, dphi, gm, &t);
  if (rc != DGPU_OK) rc = fail(c, rc, "%s", dgpu_last_error(NULL));
  /* cell_calc_cons (main.c:115) happens in dgpu_set_state */
  if (rc == DGPU_OK) rc = dgpu_set_state(c, inst, prim, tiph, dphi);
  if (rc == DGPU_OK) rc = dgpu_set_gravmass(c, inst, gm);
  if (rc == DGPU_OK) rc = dgpu_set_time(c, inst, t);
  if (rc == DGPU_OK) rc = dgpu_synchronize(c);
  free(prim); free(tiph); free(dphi);
  return rc;
}
