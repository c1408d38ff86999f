/*
 * Drop-in replacements of the reference's timestep files, on the GPU.
 *
 * A host program built from the reference's MDcode sources links
 *   activechi4_b200/legacy/cell_list_forces_b200.c  instead of cell_list+forces.c
 *   activechi4_b200/legacy/time_evolve_b200.c       instead of time_evolve.c
 * plus libactivechi4_b200.so.  The entry points keep the reference's names
 * and its calling convention (no arguments, state in the globals of
 * MDcode/global.h); the files include the program's own global.h and
 * subroutine.h.  active.c, initialise.c, print.c, main.c and Parallel.c stay
 * the reference's: direction shuffles keep the reference's host RNG stream and
 * are uploaded when they change.
 *
 * One system on one GPU: the program must run as a single MPI rank (the
 * domain decomposition of MDcode/Parallel.c is replaced by the whole system on
 * the device).  The device is CUDA device 0 unless ACG_DEVICE is set.
 */
#ifndef ACG_LEGACY_H
#define ACG_LEGACY_H

#include <stdio.h>
#include <stdlib.h>

#include "activechi4.h"

/* the engine that holds the system (created on first use from the globals)
 * for one integrator: kind 0 = Nose-Hoover NVT, 1 = NVE (advance_time_NVEFrog),
 * 2 = Berendsen NVT, 3 = Gaussian isokinetic */
acg_engine *acg_legacy_engine(int kind);
/* the engine holding the current state (the NVT engine before any step) */
acg_engine *acg_legacy_current(void);
/* host sphere[] / kx,ky,kz / thermostat globals -> device, when the host
 * changed them since the last download */
void acg_legacy_push(acg_engine *e);
/* device -> host sphere[] and the scalar globals of the step */
void acg_legacy_pull(acg_engine *e);
/* list rebuilds so far of the engine that holds the state */
long long acg_legacy_rebuilds(void);
/* print the library's last error and exit, as the reference does on errors */
void acg_legacy_die(const char *where, int rc);
/* refresh sphere[] and the step's globals from the device when it is ahead
 * (the sync points call this before the reference routine runs) */
void acg_legacy_sync_host(void);
/* host code may have edited sphere[] / the directions: compare at the next
 * device call */
void acg_legacy_host_touched(void);
void acg_legacy_dirs_touched(void);

#endif
