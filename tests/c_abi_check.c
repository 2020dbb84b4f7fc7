/* Test infrastructure: include/plfbs.h and include/plfbs_gnn.h compiled as
 * C99 and libplfbs.so called from C through entry points that need no GPU:
 * the version string, a rejected call and this thread's error message, and
 * the host cell order of a four-cell chain. tests/test_capi_host.py builds
 * and runs it; the exit status names the first failed check. */
#include <stdio.h>
#include <string.h>

#include "plfbs.h"
#include "plfbs_gnn.h"

int main(void) {
  const char* v = plfbs_version();
  if (!v || strncmp(v, "plfbs", 5) != 0) return 1;
  if (plfbs_create(NULL, NULL, NULL, NULL, 0, NULL) != PLFBS_ERR_ARG) return 2;
  if (strcmp(plfbs_last_error(NULL), "null argument") != 0) return 3;
  if (plfbs_gnn_param_count(NULL, NULL) >= 0) return 4;
  /* cells 0-1-2-3 in a chain, internal faces (1,2), (0,1), (2,3) */
  const int32_t owner[3] = {1, 0, 2}, neighbour[3] = {2, 1, 3};
  int32_t order[4] = {-1, -1, -1, -1};
  plfbs_mesh_view m;
  memset(&m, 0, sizeof m);
  m.n_cells = 4;
  m.n_faces = 3;
  m.n_internal = 3;
  m.owner = owner;
  m.neighbour = neighbour;
  if (plfbs_cell_order(&m, 0, order) != PLFBS_OK) return 5;
  for (int i = 0; i < 4; i++)
    if (order[i] != i) return 6;
  /* reverse Cuthill-McKee: start at cell 0 (degree 1, lowest index), queue
   * 0, 1, 2, 3, reversed */
  if (plfbs_cell_order(&m, 1, order) != PLFBS_OK) return 7;
  if (order[0] != 3 || order[1] != 2 || order[2] != 1 || order[3] != 0) return 8;
  if (plfbs_cell_order(&m, 3, order) != PLFBS_ERR_ARG) return 9;
  printf("%s\n", v);
  return 0;
}
