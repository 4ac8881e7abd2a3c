/*
 * pmg_mesh.h -- host-side set-up helpers of libpmg_b200 for structured
 * unit-cube problems: the data a ParMooN host would take from TDomain /
 * RegRefineAll, TFESpace3D, TSquareStructure3D and GetProlongationMatrix3D,
 * produced directly for n^3 hexahedra (Q1/Q2) or n^3 hexahedra split into six
 * Kuhn tetrahedra (P1/P2).  These run once per mesh on the host and feed
 * pmg_set_level_csr / pmg_set_level_mesh / pmg_set_transfer.
 *
 * DOF numbering: interior lattice nodes in lexicographic order (x fastest),
 * then boundary nodes, i.e. active dofs first and Dirichlet dofs last as
 * FESpace3D orders them (src/FE/FESpace3D.C:2040-2060).  Every boundary node
 * is Dirichlet (BoundCondition = DIRICHLET on all faces).
 */
#ifndef PMG_MESH_H
#define PMG_MESH_H
#ifdef __cplusplus
extern "C" {
#endif

/* sizes of a structured level: cells, dofs, local dofs per cell */
int pmg_struct_sizes(int elem_type, int n, int *n_cells, int *n_dofs, int *nloc);

/* Build the level (caller allocates): elem_dof n_cells x nloc, cell_vert
 * n_cells x 8 x 3 (tetrahedra use the first 4 vertex slots), dof_xyz N x 3,
 * dof_lat N (lattice index i + n1 (j + n1 k), n1 = degree n + 1; for N_Q1,
 * whose dofs are the 3 n^2 (n+1) faces, the face's index instead: x faces,
 * then y faces, then z faces, each i + (n_i+1)(j + ...) as the builder
 * documents).
 * jitter > 0 perturbs interior vertices by U(-jitter h, jitter h) per
 * coordinate (seeded; meaningful for tetrahedra, whose maps stay affine). */
int pmg_struct_build(int elem_type, int n, double jitter, unsigned long long seed, int *elem_dof,
                     double *cell_vert, double *dof_xyz, int *dof_lat, int *active_bound);

/* CSR pattern of TSquareStructure3D + Sort from an element->dof map:
 * kcol == NULL returns nnz in row_ptr[n_dofs] only. */
int pmg_struct_csr(int n_cells, int nloc, const int *elem_dof, int n_dofs, int active_bound, int *row_ptr,
                   int *kcol);

/* Prolongation between structured levels nc and 2 nc (interpolation on the
 * node lattice).  p_col == NULL: counts only (row_ptr filled). */
int pmg_struct_prolongation(int elem_type, int nc, const int *lat_c, int n_coarse, const int *lat_f, int n_fine,
                            int *p_row_ptr, int *p_col, double *p_val);

/* Prolongation between nested levels of any mesh: the coarse basis of the
 * coarse cell f_dof_cell[r] (a cell containing fine dof r, e.g. the parent of a
 * fine cell holding it) evaluated at fine dof r's position.  Coarse cells in the
 * pmg_set_level_mesh layout (8 vertex slots).  p_col == NULL: counts only.
 * Replaces GetProlongationMatrix3D + Prolongate (FEDatabase3D.C:1656-1815,
 * MGComponents3D.C:208-488) for conforming nested spaces. */
int pmg_nested_prolongation(int elem_type, int n_coarse_cells, const int *c_elem_dof, const double *c_cell_vert,
                            int n_coarse, int n_fine, const double *f_dof_xyz, const int *f_dof_cell,
                            int *p_row_ptr, int *p_col, double *p_val);

/* Prolongation as Prolongate applies it for any pair of spaces on nested
 * meshes (MGComponents3D.C:208-488, GetProlongationMatrix3D, FEDatabase3D.C:
 * 1656-1815): every fine cell K takes the coarse function of its parent cell
 * f_parent[K] (the cell itself when both spaces live on one mesh) at the
 * fine element's nodal points -- point values at the Lagrange nodes, at the
 * face midpoints for N_Q1 -- and every fine dof gets the mean over the fine
 * cells that hold it.  For conforming nested spaces all those values agree;
 * for N_Q1 a fine face on a coarse face takes the mean of the two parents'
 * values, and N_Q1 -> Q1 on one mesh averages the cells around a vertex.
 * Both meshes in the pmg_set_level_mesh layout (8 vertex slots per cell,
 * affine cells); p_col == NULL: counts only. */
int pmg_cell_prolongation(int c_elem_type, int n_coarse_cells, const int *c_elem_dof, const double *c_cell_vert,
                          int n_coarse, int f_elem_type, int n_fine_cells, const int *f_elem_dof,
                          const double *f_cell_vert, const int *f_parent, int n_fine, int *p_row_ptr, int *p_col,
                          double *p_val);

/* Lattice colouring for the multicolour SSOR: (i mod m, j mod m, k mod m),
 * m = degree + 1; no two coupled dofs share a colour. */
int pmg_struct_row_colors(int elem_type, int n, int n_dofs, const int *dof_lat, int *colors, int *n_colors);

#ifdef __cplusplus
}
#endif
#endif
