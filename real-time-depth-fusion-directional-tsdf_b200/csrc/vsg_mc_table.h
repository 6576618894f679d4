/* vsg_mc_table.h -- marching-cubes case table, generated from the cube's
 * geometry (plain C99; compiled into the library and into the host test
 * build).
 *
 * Numbering (the one the reference's marching-cubes kernel indexes with,
 * MarchingCubes.cu:264-285, so that case bits and interpolated vertices are
 * the same):
 *   corner k at offset (x, y, z) = ((k ^ (k >> 1)) & 1, (k >> 1) & 1, k >> 2):
 *     0 (0,0,0)  1 (1,0,0)  2 (1,1,0)  3 (0,1,0)
 *     4 (0,0,1)  5 (1,0,1)  6 (1,1,1)  7 (0,1,1)
 *   edge e joins corners kMcEdge[e][0] -> kMcEdge[e][1]; the vertex on it is
 *   interpolated from the first corner towards the second.
 *   case bit k is set when corner k's value is below the iso value ("inside").
 *
 * Triangulation rule.  On each cube face, every maximal run of inside
 * corners (taken around the face) is cut off by one segment joining the two
 * crossed edges that bound the run.  A face whose two inside corners are
 * diagonal therefore gets two segments, one around each inside corner: the
 * decision depends on the face's four corners only, so two cubes sharing a
 * face cut it identically and the surface is closed across cubes.  Segments
 * are directed from the edge where the outward face cycle leaves the run to
 * the edge where it enters it; chained over the six faces they form closed
 * loops whose triangles have cross((v1-v0),(v2-v0)) pointing towards the
 * inside corners.  Each loop is started at its smallest edge index and split
 * into a fan from that vertex, except hexagons, which are split into the
 * triangle of alternate vertices plus three ears.  At most five triangles per
 * case.
 *
 * Layout: tab[c][0..14] the edge indices of the triangles of case c, three per
 * triangle; tab[c][15] the triangle count; unused entries 0xFF.
 */
#ifndef VSG_MC_TABLE_H
#define VSG_MC_TABLE_H

#define VSG_MC_MAX_TRIS 5

static const unsigned char kMcEdge[12][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 0}, {4, 5}, {5, 6},
                                             {6, 7}, {7, 4}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};

/* The six faces as corner cycles, counter-clockwise seen from outside the
 * cube: x=0, x=1, y=0, y=1, z=0, z=1. */
static const unsigned char kMcFace[6][4] = {{4, 7, 3, 0}, {1, 2, 6, 5}, {1, 5, 4, 0},
                                            {3, 7, 6, 2}, {3, 2, 1, 0}, {4, 5, 6, 7}};

static int vsg_mc_edge_of(int a, int b) {
    int e;
    for (e = 0; e < 12; ++e)
        if ((kMcEdge[e][0] == a && kMcEdge[e][1] == b) || (kMcEdge[e][0] == b && kMcEdge[e][1] == a)) return e;
    return -1;
}

static void vsg_mc_build_table(unsigned char tab[256][16]) {
    int c, f, i, e;
    for (c = 0; c < 256; ++c) {
        int next[12];
        int done[12];
        int ntri = 0;
        for (e = 0; e < 12; ++e) {
            next[e] = -1;
            done[e] = 0;
        }
        for (i = 0; i < 16; ++i) tab[c][i] = 0xFF;
        /* face segments */
        for (f = 0; f < 6; ++f) {
            const unsigned char* cy = kMcFace[f];
            int in[4], n_in = 0;
            for (i = 0; i < 4; ++i) {
                in[i] = (c >> cy[i]) & 1;
                n_in += in[i];
            }
            if (n_in == 0 || n_in == 4) continue;
            for (i = 0; i < 4; ++i) {
                /* i starts a run: inside, previous corner outside */
                if (in[i] && !in[(i + 3) & 3]) {
                    int j = i;
                    while (in[(j + 1) & 3]) j = (j + 1) & 3;
                    {
                        const int enter = vsg_mc_edge_of(cy[(i + 3) & 3], cy[i]);
                        const int leave = vsg_mc_edge_of(cy[j], cy[(j + 1) & 3]);
                        next[leave] = enter;
                    }
                }
            }
        }
        /* loops, each from its smallest edge, then triangles */
        for (e = 0; e < 12; ++e) {
            int loop[12], n = 0, k;
            if (next[e] < 0 || done[e]) continue;
            k = e;
            do {
                loop[n++] = k;
                done[k] = 1;
                k = next[k];
            } while (k != e && n < 12);
            if (n == 6) {
                static const int ears[4][3] = {{0, 1, 2}, {2, 3, 4}, {4, 5, 0}, {0, 2, 4}};
                for (i = 0; i < 4; ++i, ++ntri) {
                    tab[c][3 * ntri + 0] = (unsigned char)loop[ears[i][0]];
                    tab[c][3 * ntri + 1] = (unsigned char)loop[ears[i][1]];
                    tab[c][3 * ntri + 2] = (unsigned char)loop[ears[i][2]];
                }
            } else {
                for (i = 1; i + 1 < n; ++i, ++ntri) {
                    tab[c][3 * ntri + 0] = (unsigned char)loop[0];
                    tab[c][3 * ntri + 1] = (unsigned char)loop[i];
                    tab[c][3 * ntri + 2] = (unsigned char)loop[i + 1];
                }
            }
        }
        tab[c][15] = (unsigned char)ntri;
    }
}

#endif /* VSG_MC_TABLE_H */
