/* timestep_gpu.c: timestep_rk2 on the B200 library, with the reference's own
 * signature (src/Headers/TimeStep.h:21). */
#ifndef TIMESTEP_GPU_H
#define TIMESTEP_GPU_H
struct TimeStep;
struct Sim;
struct Cell;
struct GravMass;
struct MPIsetup;

/* Once, after the set-up of src/main.c:56-119: the library's Sim from the
 * same parfile and a context on `device`; fused selects the fused substep.
 * Returns 0, or prints the library's message and returns its error code. */
int timestep_gpu_open(const char *parfile, int device, int fused);
/* timestep_rk2 (src/TimeStep/timestep_algorithm.c:11-41): one RK2 step of
 * the disk.  The first call uploads theCells, theGravMasses and t.  Each call
 * prints the reference's "t: %e, dt: %e" line and, unless lazy, copies the
 * new state back into theCells (prim, cons, tiph, dphi), theGravMasses (r,
 * phi, M, omega, Mdot, Macc) and theTimeStep (t, dt).  On a library error it
 * prints the message and exits, as the reference does on its own errors. */
void timestep_rk2_gpu(struct TimeStep *theTimeStep, struct Sim *theSim, struct Cell ***theCells,
                      struct GravMass *theGravMasses, struct MPIsetup *theMPIsetup);
/* lazy = 1: the state stays on the GPU between calls (t and dt still come
 * back every step); timestep_gpu_sync copies it into the reference's
 * structures when the caller needs them (diagnostics, checkpoints). */
void timestep_gpu_lazy(int lazy);
void timestep_gpu_sync(struct Sim *theSim, struct Cell ***theCells, struct GravMass *theGravMasses);
/* The next call uploads theCells, theGravMasses and t again (after the caller
 * changed them). */
void timestep_gpu_reload(void);
void timestep_gpu_close(void);
#endif
