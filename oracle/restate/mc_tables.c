/*
 * Oracle test infrastructure: marching-cubes tables derived from geometry,
 * and the marching-cubes restatement of generate_mesh_v1/v2/v3 (mesh.cpp).
 *
 * The reference's tables (marching_cubes.h:61-356) are third-party data and
 * are not copied.  Here:
 *   corners   the order mesh.cpp:19-32 samples them: 0 (0,0,0), 1 (1,0,0),
 *             2 (1,0,1), 3 (0,0,1), 4 (0,1,0), 5 (1,1,0), 6 (1,1,1), 7 (0,1,1);
 *   edges     e < 4 joins corners e and e+1 mod 4; 4 <= e < 8 joins e and
 *             4 + (e-3) mod 4; e >= 8 joins e-8 and e-4; an edge's vertex is
 *             interpolated from its lower-numbered corner a to the other, b;
 *   edge mask bit e is set when the two corners of edge e differ;
 *   polygons  on each face the active edges pair into segments; a face with
 *             four active edges separates its two corners above the iso
 *             value; segments link into loops, walked from the smallest edge
 *             towards its smaller neighbour;
 *   triangles each loop as a fan from its first edge.
 * tests/test_mesh.py checks the per-case triangle counts against the
 * reference's table (read at test time).
 */
#include "mc_tables.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

static const int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 0, 1}, {0, 0, 1},
                                  {0, 1, 0}, {1, 1, 0}, {1, 1, 1}, {0, 1, 1}};

void mc_edge_corners(int e, int *a, int *b)
{
    int p, q;
    if (e < 4) { p = e; q = (e + 1) % 4; }
    else if (e < 8) { p = e; q = 4 + (e - 3) % 4; }
    else { p = e - 8; q = e - 4; }
    *a = p < q ? p : q;
    *b = p < q ? q : p;
}

int mc_edge_mask(int c)
{
    int m = 0;
    for (int e = 0; e < 12; e++) {
        int a, b;
        mc_edge_corners(e, &a, &b);
        if (((c >> a) & 1) != ((c >> b) & 1)) m |= 1 << e;
    }
    return m;
}

/* Triangles of case c as edge triples into tri (up to 5*3 ints); returns the
 * triangle count. */
int mc_triangles(int c, int *tri)
{
    int nb[12][2], deg[12];
    for (int e = 0; e < 12; e++) deg[e] = 0;
    for (int ax = 0; ax < 3; ax++)
        for (int v = 0; v <= 1; v++) {
            int fc[4], nfc = 0;
            for (int k = 0; k < 8; k++)
                if (kCorner[k][ax] == v) fc[nfc++] = k;
            int act[4], na = 0;
            for (int e = 0; e < 12; e++) {
                int a, b;
                mc_edge_corners(e, &a, &b);
                int ina = 0, inb = 0;
                for (int q = 0; q < 4; q++) {
                    ina |= fc[q] == a;
                    inb |= fc[q] == b;
                }
                if (ina && inb && (((c >> a) & 1) != ((c >> b) & 1))) act[na++] = e;
            }
            int seg[2][2], ns = 0;
            if (na == 2) {
                seg[0][0] = act[0];
                seg[0][1] = act[1];
                ns = 1;
            } else if (na == 4) {
                for (int q = 0; q < 4; q++) {
                    const int k = fc[q];
                    if (!((c >> k) & 1)) continue;
                    int s[2], m = 0;
                    for (int i = 0; i < 4; i++) {
                        int a, b;
                        mc_edge_corners(act[i], &a, &b);
                        if (a == k || b == k) s[m++] = act[i];
                    }
                    seg[ns][0] = s[0];
                    seg[ns][1] = s[1];
                    ns++;
                }
            }
            for (int i = 0; i < ns; i++) {
                const int a = seg[i][0], b = seg[i][1];
                nb[a][deg[a]++] = b;
                nb[b][deg[b]++] = a;
            }
        }
    int visited[12] = {0};
    int nt = 0;
    for (int s = 0; s < 12; s++) {
        if (deg[s] == 0 || visited[s]) continue;
        int loop[12], n = 0;
        int prev = -1, cur = s;
        while (1) {
            loop[n++] = cur;
            visited[cur] = 1;
            int nx;
            if (prev < 0) nx = nb[cur][0] < nb[cur][1] ? nb[cur][0] : nb[cur][1];
            else nx = nb[cur][0] == prev ? nb[cur][1] : nb[cur][0];
            if (nx == s) break;
            prev = cur;
            cur = nx;
        }
        for (int i = 1; i + 1 < n; i++) {
            tri[3 * nt + 0] = loop[0];
            tri[3 * nt + 1] = loop[i];
            tri[3 * nt + 2] = loop[i + 1];
            nt++;
        }
    }
    return nt;
}

int mc_triangle_count(int c)
{
    int tri[15];
    return mc_triangles(c, tri);
}

/* Value of channel c at cube corner (x, y, z), 0 <= x <= W, 0 <= y <= H,
 * 0 <= z <= D, of a mesh snapshot with its halo as transpose_mesh_borders
 * leaves it (transposition.cpp:881-995): the +1 faces hold the periodic copy
 * of `halo` (GRID for RBB, but H for H_RB and U_SUM for U_SUM_RB, whose
 * interiors hold the previous step); halo edges and corners are never
 * written and read 0. */
static float mc_corner_value(const float *f, const float *halo, int W, int H, int c, int x, int y, int z)
{
    const int D = W;
    const int no = (x >= W) + (y >= H) + (z >= D);
    if (no > 1) return 0.0f;
    if (no == 1) f = halo;
    if (x >= W) x -= W;
    if (y >= H) y -= H;
    if (z >= D) z -= D;
    return f[(long)c * W * H * D + x + (long)y * W + (long)z * W * H];
}

void mc_own_table(int *table)
{
    for (int c = 0; c < 256; c++) {
        int tri[15];
        const int n = mc_triangles(c, tri);
        for (int k = 0; k < 16; k++) table[c * 16 + k] = k < 3 * n ? tri[k] : -1;
    }
}

/* Marching cubes with the loop order, arithmetic and vertex sharing of
 * generate_mesh_v1/v2/v3 (mesh.cpp:34-431, 434-1109, 1115-2037):
 *   - `F` fields are meshed together (v1: RBB; v2: RBB, U_SUM_RB; v3: RBB,
 *     U_SUM_RB, H_RB), each with its own vertex map (V1_EDGES, V2_EDGES,
 *     V3_EDGES), into one vertex and index buffer; per cube the fields'
 *     triangles follow each other in field order;
 *   - z is split into `slabs` ranges as the mesh threads split it
 *     (mesh.cpp:42-43); each slab has its own vertex maps (ETIDX's thread
 *     index, render.h:517) and its vertices and indices follow the previous
 *     slab's, as reset_mesh_generation concatenates them (render.cpp:161-179);
 *   - within a slab: channels, then gz, gy, gx, then fields; the vertex maps
 *     are cleared per slab, and also per channel when share == 0 (the
 *     reference clears them only per mesh, so share == 1 reproduces it);
 *   - corner i of cube g sits at (g + delta_i) * cell and is inside when its
 *     value > iso; edge vertex Pa + (Pb - Pa) * ((iso - va) / (vb - va)),
 *     then + offset[f] on each axis whose offset is nonzero (v2 and v3 shift
 *     U_SUM_RB's mesh along x and H_RB's along z by GRID_WIDTH * CELL_SIZE);
 *   - per triangle (table order) the face normal (B-A) x (C-A); each corner
 *     looks up its edge (origin, axis) in the field's vertex map, creates the
 *     vertex from this cube's position if absent, adds the face normal and
 *     appends the index.
 * fields: F pointers to C-channel fields (channel-major, x fastest); halos:
 * F pointers to the arrays the +1 halo faces copy (NULL, or a NULL entry: the
 * field itself); offset: F x 3 floats (NULL: none); table: 256 x 16 edge
 * indices, -1 terminated (NULL: mc_own_table).
 *
 * quirks != 0 reproduces how v2/v3 compute the face normals of fields 1 and
 * 2 (mesh.cpp:741, 808, 1509-1600, 1644): the fifth triangle's normal is
 * computed only when field 0 has five triangles (`tris1 == 5`), the SSE
 * path writes normal slots 0-3 from whatever the triangle slots hold, and
 * v3's scalar path for field 2 runs to field 1's triangle count.  Normal and
 * triangle slots keep their values from cube to cube within a slab, as the
 * reference's stack arrays do; a vertex whose normal used a slot never
 * written in its slab (uninitialised in the reference) is flagged in
 * `unsure`.  quirks == 0 computes every triangle's own normal.
 *
 * cases (F x C x N, optional) receives each cube's case index; vch
 * (optional) each vertex's channel + C * field; fnrm (optional, 3 floats per
 * triangle, indexed like idx) each triangle's face normal as used.  Returns
 * 0, or -1 when max_v or max_i is too small (counts are still complete). */
int ora_mesh_fields(const float *const *fields, const float *const *halos, int F, const float *offset, int W,
                    int H, int C, float iso, float cell, const int *table, int slabs, int share, int quirks,
                    unsigned char *cases, float *pos, float *nrm, int *vch, unsigned char *unsure, long max_v,
                    unsigned *idx, float *fnrm, long max_i, long *n_v, long *n_i)
{
    const int D = W;
    const long N = (long)W * H * D;
    int own[256 * 16];
    if (!table) {
        mc_own_table(own);
        table = own;
    }
    if (F < 1 || F > 3) return -1;
    const long ne = (long)(W + 1) * (H + 1) * (D + 1);
    int *emap = (int *)malloc(sizeof(int) * 3 * ne * F);
    if (!emap) return -1;
    long nv = 0, ni = 0;
    int eax[12], eo[12][3], ea[12], eb[12];
    for (int e = 0; e < 12; e++) {
        mc_edge_corners(e, &ea[e], &eb[e]);
        for (int d = 0; d < 3; d++) {
            const int ca = kCorner[ea[e]][d], cb = kCorner[eb[e]][d];
            eo[e][d] = ca < cb ? ca : cb;
            if (ca != cb) eax[e] = d;
        }
    }
    /* per field: triangle slots A, B, C and normal slots (5 x 3 floats each)
     * and whether each slot was written in this slab */
    float sv[3][3][5][3], sn[3][5][3];
    int sv_ok[3][5], sn_ok[3][5];
    memset(sv, 0, sizeof(sv));
    memset(sn, 0, sizeof(sn));
    for (int s = 0; s < slabs; s++) {
        const int z0 = (D / slabs) * s;
        const int z1 = s == slabs - 1 ? D : z0 + D / slabs;
        memset(sv_ok, 0, sizeof(sv_ok));
        memset(sn_ok, 0, sizeof(sn_ok));
        for (int c = 0; c < C; c++) {
            if (c == 0 || !share)
                for (long i = 0; i < 3 * ne * F; i++) emap[i] = -1;
            for (int gz = z0; gz < z1; gz++)
                for (int gy = 0; gy < H; gy++)
                    for (int gx = 0; gx < W; gx++) {
                        int tris0 = 0, tris1 = 0;
                        for (int f = 0; f < F; f++) {
                            const float *hf = halos && halos[f] ? halos[f] : fields[f];
                            float val[8], px[8], py[8], pz[8];
                            int cs = 0;
                            for (int i = 0; i < 8; i++) {
                                const int x = gx + kCorner[i][0], y = gy + kCorner[i][1], z = gz + kCorner[i][2];
                                val[i] = mc_corner_value(fields[f], hf, W, H, c, x, y, z);
                                px[i] = ((float)gx + (float)kCorner[i][0]) * cell;
                                py[i] = ((float)gy + (float)kCorner[i][1]) * cell;
                                pz[i] = ((float)gz + (float)kCorner[i][2]) * cell;
                                if (val[i] > iso) cs |= 1 << i;
                            }
                            if (cases)
                                cases[((long)f * C + c) * N + gx + (long)gy * W + (long)gz * W * H] = (unsigned char)cs;
                            const int emask = mc_edge_mask(cs);
                            const float ox = offset ? offset[3 * f] : 0.0f, oy = offset ? offset[3 * f + 1] : 0.0f,
                                        oz = offset ? offset[3 * f + 2] : 0.0f;
                            float vx[12], vy[12], vz[12];
                            for (int e = 0; e < 12; e++) {
                                if (!(emask & (1 << e))) continue;
                                const int a = ea[e], b = eb[e];
                                const float T = (iso - val[a]) / (val[b] - val[a]);
                                vx[e] = px[a] + (px[b] - px[a]) * T;
                                vy[e] = py[a] + (py[b] - py[a]) * T;
                                vz[e] = pz[a] + (pz[b] - pz[a]) * T;
                                if (ox != 0.0f) vx[e] = vx[e] + ox;
                                if (oy != 0.0f) vy[e] = vy[e] + oy;
                                if (oz != 0.0f) vz[e] = vz[e] + oz;
                            }
                            int *map = emap + (long)f * 3 * ne;
                            const int *tl = table + cs * 16;
                            int nt = 0;
                            while (nt < 5 && tl[3 * nt] != -1) {
                                for (int k = 0; k < 3; k++) {
                                    const int e = tl[3 * nt + k];
                                    sv[f][k][nt][0] = vx[e];
                                    sv[f][k][nt][1] = vy[e];
                                    sv[f][k][nt][2] = vz[e];
                                }
                                sv_ok[f][nt] = 1;
                                nt++;
                            }
                            if (f == 0) tris0 = nt;
                            if (f == 1) tris1 = nt;
                            /* the normal slots this cube computes: [0, hi), plus slot 4 when `fifth` */
                            int hi = nt, fifth = 0;
                            if (quirks && f > 0) {
                                if (nt >= 2) {
                                    hi = 4;
                                    fifth = tris0 == 5;
                                } else {
                                    hi = (F == 3 && f == 2) ? tris1 : nt;
                                }
                            } else if (nt == 5) {
                                hi = 4;
                                fifth = 1;
                            }
                            for (int t = 0; t < hi + fifth; t++) {
                                const int sl = t < hi ? t : 4;
                                const float *A = sv[f][0][sl], *B = sv[f][1][sl], *Cc = sv[f][2][sl];
                                const float ux = B[0] - A[0], uy = B[1] - A[1], uz = B[2] - A[2];
                                const float wx = Cc[0] - A[0], wy = Cc[1] - A[1], wz = Cc[2] - A[2];
                                sn[f][sl][0] = uy * wz - uz * wy;
                                sn[f][sl][1] = uz * wx - ux * wz;
                                sn[f][sl][2] = ux * wy - uy * wx;
                                sn_ok[f][sl] = sv_ok[f][sl];
                            }
                            for (int t = 0; t < nt; t++) {
                                const float nx = sn[f][t][0], ny = sn[f][t][1], nz = sn[f][t][2];
                                const int sure = sn_ok[f][t];
                                if (fnrm && ni < max_i) {
                                    fnrm[ni] = nx;
                                    fnrm[ni + 1] = ny;
                                    fnrm[ni + 2] = nz;
                                }
                                for (int k = 0; k < 3; k++) {
                                    const int e = tl[3 * t + k];
                                    const long ex = gx + eo[e][0], ey = gy + eo[e][1], ez = gz + eo[e][2];
                                    const long key = eax[e] * ne + ex + ey * (W + 1) + ez * (long)(W + 1) * (H + 1);
                                    int o = map[key];
                                    if (o < 0) {
                                        o = (int)nv++;
                                        map[key] = o;
                                        if (o < max_v) {
                                            pos[3 * o] = vx[e];
                                            pos[3 * o + 1] = vy[e];
                                            pos[3 * o + 2] = vz[e];
                                            nrm[3 * o] = nrm[3 * o + 1] = nrm[3 * o + 2] = 0.0f;
                                            if (vch) vch[o] = c + C * f;
                                            if (unsure) unsure[o] = 0;
                                        }
                                    }
                                    if (o < max_v) {
                                        nrm[3 * o] += nx;
                                        nrm[3 * o + 1] += ny;
                                        nrm[3 * o + 2] += nz;
                                        if (unsure && !sure) unsure[o] = 1;
                                    }
                                    if (ni < max_i) idx[ni] = (unsigned)o;
                                    ni++;
                                }
                            }
                        }
                    }
        }
    }
    free(emap);
    *n_v = nv;
    *n_i = ni;
    return (nv > max_v || ni > max_i) ? -1 : 0;
}
