/*
 * TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
 *
 * CPU oracle for PIKS3D's discrete-velocity source-iteration solver (linearised BGK,
 * binary voxel images). Only tests/, __graft_entry__.smoke() and the cpu_baseline /
 * reference leg of bench.py load this library, and only as the checker or as the timed
 * CPU baseline. The product (piks3d_b200/, libpiks3d_b200.so) never links or calls it.
 *
 * It restates, for one MPI rank of an x-only process grid (mpi_xdim ranks, mpi_ydim =
 * mpi_zdim = 1; one rank is the whole box) and in the reference's own layout f(Ntotal, Nc8,
 * 8) over the rank's ghosted box, the arithmetic of
 *   src/parameters.F90  initParams                 (:87-136)
 *   src/gaussHermite.F90 + src/velocityGrid.F90    (:90-192)
 *   src/physicalGrid.F90 setupPhysicalGrid         (:217-1625)
 *   src/flow.F90        setupFlow / allocateBuf    (:76-163)
 *   src/solver.F90      iterate                    (:111-1940)
 *   src/output.F90      chkConverge + writers      (:60-360)
 *   src/main.F90        the step loop              (:95-128)
 * with the same floating-point operation order (left-to-right sums, no FMA contraction),
 * OpenMP over the velocity index inside each octant sweep as in solver.F90:176-526.
 *
 * Parity status: UNPINNED by the reference. The reference is Fortran 90 + MPI and no
 * Fortran compiler or MPI exists in this environment, and it ships no golden vectors,
 * known-answer tests or recorded outputs. See tests/test_oracle.py for the
 * self-consistency checks that stand in for a pin.
 */
#ifndef PIKS_ORACLE_H
#define PIKS_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Namelist variables of para.in (parameters.F90:78-82), values as read, before the
 * fluidlayer / block_rep adjustments of initParams. */
typedef struct oracle_params {
  int32_t Nx, Ny, Nz, wallExtOrder, fluidlayer;
  double Ref_L;
  int32_t Nc_fundamental, halfRange;
  int32_t block_repx, block_repy, block_repz;
  int32_t maxStep, chkConvergeStep, saveStep;
  double eps;
  int32_t saveLast, saveFormat;
  double Kn, pressDrop, accom;
} oracle_params;

/* Runs initParams' adjustments, setupVelocityGrid, setupPhysicalGrid (from the raw
 * uint8 image stream, i fastest), setupFlow and allocateBuf. Returns NULL and fills
 * err on failure (invalid voxel byte, unsupported Nc_fundamental, short image). */
void *oracle_create(const oracle_params *p, const uint8_t *raw, int64_t nbytes,
                    int nthreads, char *err, int errlen);
/* The same for rank `rank` of mpi_xdim ranks along x (mpiParams.F90:150-191 with dims =
 * (mpi_xdim, 1, 1)); every rank owns at least two x planes. */
void *oracle_create_rank(const oracle_params *p, const uint8_t *raw, int64_t nbytes,
                         int nthreads, int32_t mpi_xdim, int32_t rank, char *err, int errlen);
void oracle_destroy(void *h);

/* `nsteps` calls of iterate; iStep advances by one per call. */
int oracle_iterate(void *h, int32_t nsteps);
/* chkConverge at the current iStep: updates mass/error/permeability; optionally appends
 * to results_path (Results.dat format) and prints the stdout line when verbose. */
int oracle_chk_converge(void *h, const char *results_path, int verbose, double *mass,
                        double *perm, double *err);
/* main.F90 loop: iterate/chkConverge until error <= eps or maxStep; returns steps. */
int oracle_run(void *h, const char *results_path, int verbose, int32_t *steps_out,
               double *perm_out, double *seconds_out);

/* Sizes: [Nx, Ny, Nz, Nxtotal, Nytotal, Nztotal, Ntotal, Nc8, nWall, nCorner, Nfluid,
 *         iStep, Nstencil1..8] (20 entries). */
void oracle_dims(void *h, int64_t *out);
void oracle_scalars(void *h, double *out); /* [ds, mu, DiffFlux, mass, error, permeability] */
void oracle_velocity(void *h, double *cx, double *cy, double *cz, double *w);
void oracle_get_image(void *h, int32_t *out);        /* ghosted image, Ntotal, i fastest */
void oracle_get_which_corner(void *h, int32_t *out); /* ghosted, Ntotal */
void oracle_get_vecwall(void *h, int32_t *out);      /* nWall local ids (1-based) */
void oracle_get_mapf(void *h, int32_t *out);         /* Nfluid local ids (1-based) */
void oracle_get_extcoef(void *h, double *out);       /* nWall x 2, column-major */
void oracle_get_f(void *h, double *out);             /* Ntotal x Nc8 x 8, column-major */
void oracle_set_f(void *h, const double *in);
void oracle_get_f_at(void *h, const int64_t *gidx, int32_t n, double *out); /* n x 8 x Nc8 rows at ghosted indices */
void oracle_get_fw(void *h, double *out);            /* nCorner x Nc8 x 8 */
void oracle_get_macro(void *h, double *rho, double *ux, double *uy, double *uz); /* Ntotal */
void oracle_get_dir(void *h, int octant, int32_t *out);   /* 3 x Nstencil */
void oracle_get_coef(void *h, int octant, double *out);   /* Nstencil x 9 */

/* Field writers of output.F90 (VTI/VTK/Tecplot, proc 000) into directory `dir`. */
int oracle_save(void *h, const char *dir, int format);

/* [xl, xu, xlg, mpi_xdim, rank] of the rank's slab (global 1-based x). */
void oracle_slab(void *h, int32_t *out);
/* x messages of solver.F90:146-170 / :535-612 (the face part, oracle_halo_size doubles
 * each): oracle_halo_send copies out the buffers the last iteration packed (what the rank
 * sends west / east at the start of the next one); oracle_halo_recv sets what it receives
 * from its west / east neighbour for the next iteration. With mpi_xdim = 1 iterate moves
 * them itself. */
int64_t oracle_halo_size(void *h);
void oracle_halo_send(void *h, double *west, double *east);
void oracle_halo_recv(void *h, const double *west, const double *east);
/* Setters of the rest of the iteration state (for tests that move the state: fw as
 * oracle_get_fw, the macro fields as oracle_get_macro, the packed x messages). */
void oracle_set_fw(void *h, const double *in);
void oracle_set_macro(void *h, const double *rho, const double *ux, const double *uy, const double *uz);
void oracle_set_halo_send(void *h, const double *west, const double *east);

#ifdef __cplusplus
}
#endif
#endif
