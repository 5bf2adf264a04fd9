// ORACLE — TEST INFRASTRUCTURE ONLY.
// Single-process stand-in for the two ParMETIS 3.x calls in Free CFD's grid
// setup (grid/grid_partition.cc).  With one rank every cell belongs to
// partition 0, and the dual graph is only read for faces next to another
// partition (grid_create_elements.cc:561-650 runs that loop for np > 1 only),
// so it is returned empty.
#ifndef FCFD_REF_STUB_PARMETIS_H
#define FCFD_REF_STUB_PARMETIS_H

#include "mpi.h"

typedef int idxtype;

static inline int ParMETIS_V3_PartMeshKway(idxtype *elmdist, idxtype *, idxtype *, idxtype *, int *, int *, int *,
                                           int *, int *nparts, float *, float *, int *, int *edgecut, idxtype *part,
                                           MPI_Comm *) {
  const int n = elmdist[1] - elmdist[0];
  for (int c = 0; c < n; ++c) part[c] = 0;
  (void)nparts;
  *edgecut = 0;
  return 0;
}

static inline int ParMETIS_V3_Mesh2Dual(idxtype *elmdist, idxtype *, idxtype *, int *, int *, idxtype **xadj,
                                        idxtype **adjncy, MPI_Comm *) {
  const int n = elmdist[1] - elmdist[0];
  *xadj = new idxtype[n + 1]();
  *adjncy = new idxtype[1]();
  return 0;
}

#endif
