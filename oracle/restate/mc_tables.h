/* Oracle test infrastructure: marching-cubes tables and restatement
 * (mc_tables.c). */
#ifndef LENIA_ORACLE_MC_TABLES_H
#define LENIA_ORACLE_MC_TABLES_H

#ifdef __cplusplus
extern "C" {
#endif

void mc_edge_corners(int e, int *a, int *b);
int mc_edge_mask(int c);
int mc_triangles(int c, int *tri);
int mc_triangle_count(int c);
void mc_own_table(int *table);
int ora_mesh_fields(const float *const *fields, const float *const *halos, int F, const float *offset, int W,
                    int H, int C, float iso, float cell, const int *table, int slabs, int share, int quirks,
                    unsigned char *cases, float *pos, float *nrm, int *vch, unsigned char *unsure, long max_v,
                    unsigned *idx, float *fnrm, long max_i, long *n_v, long *n_i);

#ifdef __cplusplus
}
#endif
#endif
