/*
 * cell_list+forces.c on the GPU: update_cell_list and calculate_forces run on
 * the device (acg_rebuild, acg_compute_forces); getcell_I, maps and len_check
 * are the reference's small host utilities (MDcode/cell_list+forces.c:24-54,
 * 229-244), still called by the reference's Parallel.c.
 *
 * The device keeps its own neighbour lists: NeibList/NeibListCount are not
 * filled.  InCell/InCellCount are filled from the device's cell list (same
 * cells, same ascending order inside a cell).
 */
#include "acg_legacy.h" /* before global.h, whose macros (skin) clash with field names */
#include "global.h"
#include "subroutine.h"

static double sigma_[3][3] = {{1.00, 0.80, 1.0}, {0.80, 0.88, 1.0}, {1.0, 1.0, 1.0}};

int getcell_I(int Ix, int Iy, int Iz) {
  return ((Ix + Ncellx * 3) % Ncellx) + ((Iy + Ncelly * 3) % Ncelly) * Ncellx +
         ((Iz + Ncellz * 3) % Ncellz) * Ncellx * Ncelly;
}

void maps() {
  static const int off[13][3] = {{1, 0, 0},  {1, 1, 0},  {0, 1, 0},  {-1, 1, 0}, {1, 0, -1},
                                 {1, 1, -1}, {0, 1, -1}, {-1, 1, -1}, {1, 0, 1}, {1, 1, 1},
                                 {0, 1, 1},  {-1, 1, 1}, {0, 0, 1}};
  for (int Ix = 0; Ix < Ncellx; Ix++)
    for (int Iy = 0; Iy < Ncelly; Iy++)
      for (int Iz = 0; Iz < Ncellz; Iz++) {
        int c = getcell_I(Ix, Iy, Iz);
        for (int m = 0; m < 13; m++) MAP[c][m] = getcell_I(Ix + off[m][0], Iy + off[m][1], Iz + off[m][2]);
      }
}

bool len_check(SPHERE s1, SPHERE s2) {
  double dx = s1.x - s2.x, dy = s1.y - s2.y, dz = s1.z - s2.z;
  if (dx < -HALF_LENGTH) dx += LENGTH;
  if (dx > HALF_LENGTH) dx -= LENGTH;
  if (dy < -HALF_LENGTH) dy += LENGTH;
  if (dy > HALF_LENGTH) dy -= LENGTH;
  if (dz < -HALF_LENGTH) dz += LENGTH;
  if (dz > HALF_LENGTH) dz -= LENGTH;
  double dr2 = (dx * dx + dy * dy + dz * dz) * L * L;
  double sig = sigma_[s1.type][s2.type];
  return dr2 / (sig * sig) < Cell_cut_sq;
}

/* update_cell_list (MDcode/cell_list+forces.c:58-148) */
void update_cell_list() {
  acg_engine *e = acg_legacy_current();
  acg_legacy_sync_host(); /* xold below is taken from sphere[] */
  acg_legacy_push(e);
  int rc = acg_rebuild(e);
  if (rc) acg_legacy_die("acg_rebuild", rc);
  int dims[3], ncell = 0;
  rc = acg_get_cells(e, 0, dims, &ncell, NULL, NULL);
  if (rc) acg_legacy_die("acg_get_cells", rc);
  int *counts = (int *)malloc(sizeof(int) * (size_t)ncell), *members = (int *)malloc(sizeof(int) * N);
  if (!counts || !members) {
    fprintf(stderr, "activechi4: host allocation failed\n");
    exit(1);
  }
  rc = acg_get_cells(e, 0, dims, &ncell, counts, members);
  if (rc) acg_legacy_die("acg_get_cells", rc);
  int m = 0;
  for (int c = 0; c < ncell && c < MaxCells; c++) {
    InCellCount[c] = counts[c];
    for (int j = 0; j < counts[c]; j++, m++)
      if (j < MaxPartInCell) InCell[c][j] = members[m];
  }
  free(counts);
  free(members);
  for (int i = 0; i < N; i++) {
    xold[i] = sphere[i].x_u;
    yold[i] = sphere[i].y_u;
    zold[i] = sphere[i].z_u;
  }
  maxD = 0.0;
  globalMaxD = 0.0;
}

/* calculate_forces (MDcode/cell_list+forces.c:153-227): pair + active forces,
 * pe, virial and vir_act of the whole system */
void calculate_forces() {
  acg_engine *e = acg_legacy_current();
  acg_legacy_push(e);
  int rc = acg_compute_forces(e);
  if (rc) acg_legacy_die("acg_compute_forces", rc);
  acg_legacy_pull(e);
}
