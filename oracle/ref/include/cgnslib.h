// ORACLE — TEST INFRASTRUCTURE ONLY.
// Declarations that let grid/grid_reader_cgns.cc compile without libcgns.
// Every call reports an error: the harness feeds grids through the
// reference's own raw grid file (Grid::read_raw, grid_reader_cgns.cc:433-489)
// and never reaches the CGNS reader.
#ifndef FCFD_REF_STUB_CGNSLIB_H
#define FCFD_REF_STUB_CGNSLIB_H

#define CG_OK 0
#define CG_ERROR 1
#define MODE_READ 0

enum ElementType_t { ElementTypeNull, ElementTypeUserDefined, NODE, BAR_2, BAR_3, TRI_3, TRI_6, QUAD_4, QUAD_8, QUAD_9,
                     TETRA_4, TETRA_10, PYRA_5, PYRA_14, PENTA_6, PENTA_15, PENTA_18, HEXA_8, HEXA_20, HEXA_27,
                     MIXED, NGON_n };
enum BCType_t { BCTypeNull };
enum PointSetType_t { PointSetTypeNull, PointSetTypeUserDefined, PointList, PointListDonor, PointRange, PointRangeDonor,
                      ElementRange, ElementList, CellListDonor };
enum DataType_t { DataTypeNull, DataTypeUserDefined, Integer, RealSingle, RealDouble, Character };
enum ZoneType_t { ZoneTypeNull };

static inline int cg_open(...) { return CG_ERROR; }
static inline int cg_nbases(...) { return CG_ERROR; }
static inline int cg_nzones(...) { return CG_ERROR; }
static inline int cg_zone_read(...) { return CG_ERROR; }
static inline int cg_nsections(...) { return CG_ERROR; }
static inline int cg_nbocos(...) { return CG_ERROR; }
static inline int cg_boco_info(...) { return CG_ERROR; }
static inline int cg_boco_read(...) { return CG_ERROR; }
static inline int cg_section_read(...) { return CG_ERROR; }
static inline int cg_ElementDataSize(...) { return CG_ERROR; }
static inline int cg_elements_read(...) { return CG_ERROR; }
static inline int cg_coord_read(...) { return CG_ERROR; }
static inline int cg_npe(...) { return CG_ERROR; }

#endif
