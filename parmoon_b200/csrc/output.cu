// VTK output of a level's finite-element function, written from the device
// (TOutput3D::WriteVtk, src/FE/Output3D.C:1773-2292).
//
// The reference numbers the distinct vertices of the collection, writes their
// coordinates, the cells by vertex number (VTK_HEXAHEDRON = 12, VTK_TETRA = 10,
// corners in the cell's own vertex order), and as POINT_DATA the function
// evaluated at every cell corner, averaged over the cells that share the
// vertex, then the cells' region ids as CELL_DATA.  For the Lagrange
// elements here every vertex is a node: the value at corner j of a cell is the
// coefficient of the local node sitting there, the same in every cell.  So the
// vertices are the corner nodes, numbered in dof order: one kernel marks them,
// gathers their coordinates from the cells and their values from the
// device-resident vector; the host only numbers the marked dofs and formats
// the file (the reference's ASCII layout, values in scientific notation with
// 6 digits after the point).
#include "pmg_internal.h"
#include "fe_tables.h"
#include <cstdio>
#include <vector>

namespace pmg {

// local node at VTK corner j: hexahedra (-1,-1,-1), (1,-1,-1), (1,1,-1),
// (-1,1,-1), then z = +1; tetrahedra the four vertices (the reference's
// HexaCoords / TetraCoords, Output3D.C:1816-1834)
static const int kCornerQ1[8] = {0, 1, 3, 2, 4, 5, 7, 6};
static const int kCornerQ2[8] = {0, 2, 8, 6, 18, 20, 26, 24};
static const int kCornerP1[4] = {0, 1, 2, 3};
static const int kCornerP2[4] = {0, 2, 5, 9};

struct Corners {
  int c[8];
};

__global__ void k_vtk_corners(int n_cells, int nloc, int nv, Corners corner, const int *__restrict__ elem_dof,
                              const double *__restrict__ cell_vert, const double *__restrict__ u,
                              double *__restrict__ xyzv, unsigned char *__restrict__ is_vertex) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long)n_cells * nv) return;
  const int e = (int)(t / nv), j = (int)(t % nv);
  const int d = elem_dof[(size_t)e * nloc + corner.c[j]];
  // every cell sharing the vertex writes the same coordinates and value
  is_vertex[d] = 1;
  const double *cv = cell_vert + ((size_t)e * nv + j) * 3;
  xyzv[(size_t)d * 4 + 0] = cv[0];
  xyzv[(size_t)d * 4 + 1] = cv[1];
  xyzv[(size_t)d * 4 + 2] = cv[2];
  xyzv[(size_t)d * 4 + 3] = u[d];
}

}  // namespace pmg

using namespace pmg;

extern "C" int pmg_write_vtk(pmg_handle hh, int level, const double *values, const int *region_ids, const char *path,
                             const char *name) {
  Handle *h = reinterpret_cast<Handle *>(hh);
  if (!h || level < 0 || level >= (int)h->lv.size() || !path || !name || !name[0]) {
    set_error("pmg_write_vtk: bad arguments");
    return PMG_ERR_ARG;
  }
  for (const char *c = name; *c; c++)
    if (*c == ' ' || *c == '\n' || *c == '\t') {
      set_error("pmg_write_vtk: the field name must not contain white space (VTK keyword syntax)");
      return PMG_ERR_ARG;
    }
  Level &L = h->lv[level];
  if (!L.has_mesh) {
    set_error("pmg_write_vtk: the level has no mesh (pmg_set_level_mesh)");
    return PMG_ERR_STATE;
  }
  if (L.elem == PMG_ELEM_NQ1_HEX) {
    set_error("pmg_write_vtk: N_Q1 has no nodes at the cell corners (write the conforming level)");
    return PMG_ERR_UNSUPPORTED;
  }
  const double *u = nullptr;
  DBuf<double> du;
  if (values) {
    PMG_TRY(du.upload(values, L.N, h->stream));
    u = du.p;
  } else {
    if (level != (int)h->lv.size() - 1 || !h->sol.p || h->sol.n < (size_t)L.N) {
      set_error("pmg_write_vtk: no device-resident solution of this level (pmg_solve first, or pass values)");
      return PMG_ERR_STATE;
    }
    u = h->sol.p;
  }
  const bool hex = elem_is_hex(L.elem);
  const int nv = hex ? 8 : 4;
  Corners corner{};
  const int *cm = L.elem == PMG_ELEM_Q1_HEX ? kCornerQ1
                : L.elem == PMG_ELEM_Q2_HEX ? kCornerQ2
                : L.elem == PMG_ELEM_P1_TET ? kCornerP1 : kCornerP2;
  for (int j = 0; j < nv; j++) corner.c[j] = cm[j];
  DBuf<double> xyzv;
  DBuf<unsigned char> mark;
  PMG_TRY(xyzv.alloc((size_t)L.N * 4));
  PMG_TRY(mark.alloc(L.N));
  PMG_CUDA(cudaMemsetAsync(mark.p, 0, L.N, h->stream));
  const long work = (long)L.n_cells * nv;
  k_vtk_corners<<<(unsigned)((work + 255) / 256), 256, 0, h->stream>>>(L.n_cells, L.nloc, nv, corner, L.elem_dof.p,
                                                                        L.cell_vert.p, u, xyzv.p, mark.p);
  count_launches(1);
  PMG_CUDA(cudaGetLastError());
  std::vector<double> hx((size_t)L.N * 4);
  std::vector<unsigned char> hm(L.N);
  std::vector<int> ed((size_t)L.n_cells * L.nloc);
  PMG_CUDA(cudaMemcpyAsync(hx.data(), xyzv.p, sizeof(double) * hx.size(), cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaMemcpyAsync(hm.data(), mark.p, hm.size(), cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaMemcpyAsync(ed.data(), L.elem_dof.p, sizeof(int) * ed.size(), cudaMemcpyDeviceToHost, h->stream));
  PMG_CUDA(cudaStreamSynchronize(h->stream));
  // vertex numbers in dof order
  std::vector<int> vid(L.N, -1);
  int nvert = 0;
  for (int d = 0; d < L.N; d++)
    if (hm[d]) vid[d] = nvert++;
  FILE *f = fopen(path, "w");
  if (!f) {
    set_error(std::string("pmg_write_vtk: cannot open ") + path);
    return PMG_ERR_ARG;
  }
  fprintf(f, "# vtk DataFile Version 4.2\nfile created by ParMooN\nASCII\nDATASET UNSTRUCTURED_GRID\n\n");
  fprintf(f, "POINTS %d double\n", nvert);
  for (int d = 0; d < L.N; d++)
    if (hm[d]) fprintf(f, "%e %e %e\n", hx[(size_t)d * 4], hx[(size_t)d * 4 + 1], hx[(size_t)d * 4 + 2]);
  fprintf(f, "\nCELLS %d %ld\n", L.n_cells, (long)L.n_cells * (nv + 1));
  // cells in the caller's order (the device keeps them in element-colour order)
  std::vector<int> pos(L.n_cells);
  for (int k = 0; k < L.n_cells; k++) pos[L.cell_order[k]] = k;
  for (int c = 0; c < L.n_cells; c++) {
    const int *dof = ed.data() + (size_t)pos[c] * L.nloc;
    fprintf(f, "%d ", nv);
    for (int j = 0; j < nv; j++) fprintf(f, "%d ", vid[dof[cm[j]]]);
    fprintf(f, "\n");
  }
  fprintf(f, "\nCELL_TYPES %d\n", L.n_cells);
  for (int c = 0; c < L.n_cells; c++) fprintf(f, "%d ", hex ? 12 : 10);
  fprintf(f, "\n\nPOINT_DATA %d\n", nvert);
  fprintf(f, "SCALARS %s double\nLOOKUP_TABLE default\n", name);
  for (int d = 0; d < L.N; d++)
    if (hm[d]) fprintf(f, "%e\n", hx[(size_t)d * 4 + 3]);
  fprintf(f, "\n");
  // the cells' region ids as CELL_DATA (Output3D.C:2282-2292)
  fprintf(f, "\nCELL_DATA %d\nSCALARS RegionID int  1\nLOOKUP_TABLE default  \n", L.n_cells);
  for (int c = 0; c < L.n_cells; c++) fprintf(f, "%d\n", region_ids ? region_ids[c] : 0);
  const bool ok = ferror(f) == 0;
  fclose(f);
  if (!ok) {
    set_error(std::string("pmg_write_vtk: write error on ") + path);
    return PMG_ERR_ARG;
  }
  return PMG_OK;
}
