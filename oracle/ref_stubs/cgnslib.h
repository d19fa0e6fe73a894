/* In-memory CGNS stand-in used only to compile the reference's CPU path as a
 * test checker (oracle/_ref). It serves the ~20 read calls that the
 * reference's Mesh2D_t::read_cgns makes (src/meshes/Mesh2D_t.cpp:422-1048)
 * from one unstructured zone held in `ndg_mem_cgns`, which the checker's
 * driver fills before constructing a mesh. Any file name is accepted: the
 * zone is never read from disk. Test infrastructure only. */
#ifndef NDG_ORACLE_STUB_CGNSLIB_H
#define NDG_ORACLE_STUB_CGNSLIB_H

#include <cstring>
#include <string>
#include <vector>

typedef long cgsize_t;

#define CG_OK 0
#define CG_ERROR 1
#define CG_MODE_READ 0
#define CG_MODE_WRITE 1

enum ZoneType_t { ZoneTypeNull = 0, ZoneTypeUserDefined, Structured, Unstructured };
enum DataType_t { DataTypeNull = 0, DataTypeUserDefined, Integer, RealSingle, RealDouble, Character, LongInteger };
enum ElementType_t { ElementTypeNull = 0, ElementTypeUserDefined, NODE, BAR_2, BAR_3, TRI_3, TRI_6, QUAD_4 };
enum GridLocation_t { GridLocationNull = 0, GridLocationUserDefined, Vertex, CellCenter, FaceCenter, IFaceCenter, JFaceCenter, KFaceCenter, EdgeCenter };
enum GridConnectivityType_t { GridConnectivityTypeNull = 0, GridConnectivityTypeUserDefined, Overset, Abutting, Abutting1to1 };
enum PointSetType_t { PointSetTypeNull = 0, PointSetTypeUserDefined, PointList, PointListDonor, PointRange, PointRangeDonor, ElementRange, ElementList, CellListDonor };
enum BCType_t { BCTypeNull = 0, BCTypeUserDefined, BCInflow, BCOutflow, BCSymmetryPlane, BCWall };

struct NdgMemSection {
    std::string name;
    ElementType_t type;
    cgsize_t start;
    cgsize_t end;
    std::vector<cgsize_t> connectivity; /* 1-based node indices */
};

struct NdgMemBoco {
    std::string name;
    BCType_t type;
    std::vector<cgsize_t> points; /* 1-based element indices */
};

struct NdgMemConn {
    std::string name;
    std::vector<cgsize_t> points;       /* 1-based element indices */
    std::vector<cgsize_t> donor_points; /* 1-based element indices, same zone */
};

struct NdgMemZone {
    std::string zone_name{"Zone 1"};
    std::vector<double> x;
    std::vector<double> y;
    std::vector<NdgMemSection> sections;
    std::vector<NdgMemBoco> bocos;
    std::vector<NdgMemConn> conns;
};

extern NdgMemZone ndg_mem_cgns;

inline void ndg_mem_copy_name(char* dst, const std::string& src) {
    std::strncpy(dst, src.c_str(), 32);
    dst[32] = '\0';
}

inline int cg_open(const char*, int, int* fn) { *fn = 1; return CG_OK; }
inline int cg_close(int) { return CG_OK; }
inline const char* cg_get_error() { return "in-memory zone"; }
inline int cg_nbases(int, int* n) { *n = 1; return CG_OK; }
inline int cg_base_read(int, int, char* name, int* cell_dim, int* phys_dim) {
    ndg_mem_copy_name(name, "Base");
    *cell_dim = 2;
    *phys_dim = 2;
    return CG_OK;
}
inline int cg_nzones(int, int, int* n) { *n = 1; return CG_OK; }
inline int cg_zone_read(int, int, int, char* name, cgsize_t* size) {
    ndg_mem_copy_name(name, ndg_mem_cgns.zone_name);
    cgsize_t n_elements = 0;
    for (const auto& s : ndg_mem_cgns.sections) {
        n_elements += s.end - s.start + 1;
    }
    size[0] = static_cast<cgsize_t>(ndg_mem_cgns.x.size());
    size[1] = n_elements;
    size[2] = 0;
    return CG_OK;
}
inline int cg_zone_type(int, int, int, ZoneType_t* t) { *t = Unstructured; return CG_OK; }
inline int cg_ncoords(int, int, int, int* n) { *n = 2; return CG_OK; }
inline int cg_coord_info(int, int, int, int c, DataType_t* t, char* name) {
    *t = RealDouble;
    ndg_mem_copy_name(name, c == 1 ? "CoordinateX" : "CoordinateY");
    return CG_OK;
}
inline int cg_coord_read(int, int, int, const char* name, DataType_t, const cgsize_t* rmin, const cgsize_t* rmax, void* out) {
    const std::vector<double>& src = (std::strcmp(name, "CoordinateX") == 0) ? ndg_mem_cgns.x : ndg_mem_cgns.y;
    double* dst = static_cast<double*>(out);
    for (cgsize_t i = *rmin; i <= *rmax; ++i) {
        dst[i - *rmin] = src[static_cast<size_t>(i - 1)];
    }
    return CG_OK;
}
inline int cg_nsections(int, int, int, int* n) { *n = static_cast<int>(ndg_mem_cgns.sections.size()); return CG_OK; }
inline int cg_ElementDataSize(int, int, int, int s, cgsize_t* size) {
    *size = static_cast<cgsize_t>(ndg_mem_cgns.sections[static_cast<size_t>(s - 1)].connectivity.size());
    return CG_OK;
}
inline int cg_section_read(int, int, int, int s, char* name, ElementType_t* type, cgsize_t* start, cgsize_t* end, int* nbndry, int* parent_flag) {
    const NdgMemSection& sec = ndg_mem_cgns.sections[static_cast<size_t>(s - 1)];
    ndg_mem_copy_name(name, sec.name);
    *type = sec.type;
    *start = sec.start;
    *end = sec.end;
    *nbndry = 0;
    *parent_flag = 0;
    return CG_OK;
}
inline int cg_elements_read(int, int, int, int s, cgsize_t* elements, cgsize_t*) {
    const NdgMemSection& sec = ndg_mem_cgns.sections[static_cast<size_t>(s - 1)];
    std::memcpy(elements, sec.connectivity.data(), sec.connectivity.size() * sizeof(cgsize_t));
    return CG_OK;
}
inline int cg_nconns(int, int, int, int* n) { *n = static_cast<int>(ndg_mem_cgns.conns.size()); return CG_OK; }
inline int cg_conn_info(int, int, int, int i, char* name, GridLocation_t* location, GridConnectivityType_t* type, PointSetType_t* ptset_type, cgsize_t* npnts, char* donorname, ZoneType_t* donor_zonetype, PointSetType_t* donor_ptset_type, DataType_t* donor_datatype, cgsize_t* ndata_donor) {
    const NdgMemConn& c = ndg_mem_cgns.conns[static_cast<size_t>(i - 1)];
    ndg_mem_copy_name(name, c.name);
    *location = FaceCenter;
    *type = Abutting1to1;
    *ptset_type = PointList;
    *npnts = static_cast<cgsize_t>(c.points.size());
    std::memset(donorname, 0, 33);
    ndg_mem_copy_name(donorname, ndg_mem_cgns.zone_name);
    *donor_zonetype = Unstructured;
    *donor_ptset_type = PointListDonor;
    *donor_datatype = Integer;
    *ndata_donor = static_cast<cgsize_t>(c.donor_points.size());
    return CG_OK;
}
inline int cg_conn_read(int, int, int, int i, cgsize_t* pnts, DataType_t, cgsize_t* donor_data) {
    const NdgMemConn& c = ndg_mem_cgns.conns[static_cast<size_t>(i - 1)];
    std::memcpy(pnts, c.points.data(), c.points.size() * sizeof(cgsize_t));
    std::memcpy(donor_data, c.donor_points.data(), c.donor_points.size() * sizeof(cgsize_t));
    return CG_OK;
}
inline int cg_nbocos(int, int, int, int* n) { *n = static_cast<int>(ndg_mem_cgns.bocos.size()); return CG_OK; }
inline int cg_boco_info(int, int, int, int bc, char* name, BCType_t* type, PointSetType_t* ptset_type, cgsize_t* npnts, int* normal_index, cgsize_t* normal_list_size, DataType_t* normal_data_type, int* ndataset) {
    const NdgMemBoco& b = ndg_mem_cgns.bocos[static_cast<size_t>(bc - 1)];
    ndg_mem_copy_name(name, b.name);
    *type = b.type;
    *ptset_type = PointList;
    *npnts = static_cast<cgsize_t>(b.points.size());
    normal_index[0] = 0;
    *normal_list_size = 0;
    *normal_data_type = DataTypeNull;
    *ndataset = 0;
    return CG_OK;
}
inline int cg_boco_gridlocation_read(int, int, int, int, GridLocation_t* location) { *location = EdgeCenter; return CG_OK; }
inline int cg_boco_read(int, int, int, int bc, cgsize_t* pnts, void*) {
    const NdgMemBoco& b = ndg_mem_cgns.bocos[static_cast<size_t>(bc - 1)];
    std::memcpy(pnts, b.points.data(), b.points.size() * sizeof(cgsize_t));
    return CG_OK;
}

#endif
