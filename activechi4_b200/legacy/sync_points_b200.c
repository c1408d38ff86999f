/*
 * Sync points of the drop-in: the reference routines (kept as the program's
 * own, in Parallel.c, initialise.c, print.c and active.c) that read or write
 * sphere[] or the direction arrays.  Linking with
 *
 *   -Wl,--wrap=GatherCoordinatesToRoot,--wrap=GatherCoordAndMomentaToRoot,
 *   -Wl,--wrap=ExchangeParticlesInBlocks,--wrap=CommunicateCoordinates,
 *   -Wl,--wrap=BcastInitState,--wrap=SetUpParallel,--wrap=fixDrift,
 *   -Wl,--wrap=calculate_temp,--wrap=adjustInitialTemp,--wrap=print_stuff,
 *   -Wl,--wrap=print_eq,--wrap=print_movie,--wrap=ShuffleActDirec,
 *   -Wl,--wrap=readActiveDirection,--wrap=readActiveParticles,
 *   -Wl,--wrap=selectRandomActiveParticles
 *
 * sends the program's calls of these routines (from other files: main.c's
 * run loop and restart writer, print.c) through the wrappers below, which
 * refresh sphere[] from the device first when the device is ahead
 * (write_restart_state and print_data read sphere[] after their Gather*
 * call) and note that the host may have changed the state afterwards.  The
 * step itself (AdvanceTimeNVTNoseHoover) then moves no particle data between
 * host and device.
 */
#include "acg_legacy.h" /* before global.h, whose macros (skin) clash with field names */
#include "global.h"
#include "subroutine.h"

#define SYNC_VOID(name)             \
  void __real_##name(void);         \
  void __wrap_##name(void) {        \
    acg_legacy_sync_host();         \
    __real_##name();                \
    acg_legacy_host_touched();      \
  }

SYNC_VOID(GatherCoordinatesToRoot)
SYNC_VOID(GatherCoordAndMomentaToRoot)
SYNC_VOID(ExchangeParticlesInBlocks)
SYNC_VOID(BcastInitState)
SYNC_VOID(SetUpParallel)
SYNC_VOID(fixDrift)
SYNC_VOID(calculate_temp)
SYNC_VOID(selectRandomActiveParticles)

void __real_CommunicateCoordinates(int refill);
void __wrap_CommunicateCoordinates(int refill) {
  acg_legacy_sync_host();
  __real_CommunicateCoordinates(refill);
  acg_legacy_host_touched();
}

void __real_adjustInitialTemp(double final_temp);
void __wrap_adjustInitialTemp(double final_temp) {
  acg_legacy_sync_host();
  __real_adjustInitialTemp(final_temp);
  acg_legacy_host_touched();
}

double __real_print_stuff(char infile[]);
double __wrap_print_stuff(char infile[]) {
  acg_legacy_sync_host();
  return __real_print_stuff(infile);
}

double __real_print_eq(char infile1[]);
double __wrap_print_eq(char infile1[]) {
  acg_legacy_sync_host();
  return __real_print_eq(infile1);
}

double __real_print_movie(void);
double __wrap_print_movie(void) {
  acg_legacy_sync_host();
  return __real_print_movie();
}

/* direction arrays: host-owned (ShuffleActDirec keeps the program's RNG);
 * uploaded at the next device call when they changed */
void __real_ShuffleActDirec(void);
void __wrap_ShuffleActDirec(void) {
  __real_ShuffleActDirec();
  acg_legacy_dirs_touched();
}

void __real_readActiveDirection(char *inFileName);
void __wrap_readActiveDirection(char *inFileName) {
  __real_readActiveDirection(inFileName);
  acg_legacy_dirs_touched();
}

void __real_readActiveParticles(char *activeFile);
void __wrap_readActiveParticles(char *activeFile) {
  acg_legacy_sync_host();
  __real_readActiveParticles(activeFile);
  acg_legacy_host_touched();
}
