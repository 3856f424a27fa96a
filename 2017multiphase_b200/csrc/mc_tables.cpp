// mc_tables.cpp — marching-cubes case tables, generated.
//
// The reference reads the classic Lorensen/Bourke tables from tables.h
// (Multiphase/Multiphase/tables.h:19-575). They are not copied here; they are
// built from first principles with the same conventions the reference's
// kernels assume (spray_k.cu:1853-2170):
//   corner v has bit v of the case index set when its field value is below
//   the iso value; corners v0..v7 = (0,0,0) (1,0,0) (1,1,0) (0,1,0)
//   (0,0,1) (1,0,1) (1,1,1) (0,1,1); edges 0..11 join corners
//   0-1 1-2 2-3 3-0 4-5 5-6 6-7 7-4 0-4 1-5 2-6 3-7.
// Construction: on each cube face, connect the crossing points of its edges
// into segments oriented so that the set corners lie to the left as seen
// from outside; on a face with two diagonal set corners each set corner is
// cut off by its own segment. With that rule every case has the classic
// table's triangle count and the same crossed edges (checked against
// tables.h by tests/test_mc_tables.py). The segments close into loops, and
// each loop is fanned into triangles from its lowest edge. Triangle normals
// (right-hand rule) point towards the set corners, as in the classic table.
#include <cstdint>
#include <cstring>
#include <vector>
#include <algorithm>

namespace {

const int kCorner[8][3] = {{0,0,0},{1,0,0},{1,1,0},{0,1,0},{0,0,1},{1,0,1},{1,1,1},{0,1,1}};
const int kEdge[12][2] = {{0,1},{1,2},{2,3},{3,0},{4,5},{5,6},{6,7},{7,4},{0,4},{1,5},{2,6},{3,7}};
// faces as cyclic corner lists with their outward normals
const int kFace[6][4] = {{0,1,2,3},{4,5,6,7},{0,1,5,4},{3,2,6,7},{0,3,7,4},{1,2,6,5}};
const int kNormal[6][3] = {{0,0,-1},{0,0,1},{0,-1,0},{0,1,0},{-1,0,0},{1,0,0}};

int edge_of(int a, int b) {
    for (int e = 0; e < 12; e++)
        if ((kEdge[e][0] == a && kEdge[e][1] == b) || (kEdge[e][0] == b && kEdge[e][1] == a)) return e;
    return -1;
}
void mid(int e, double m[3]) {
    for (int q = 0; q < 3; q++) m[q] = 0.5 * (kCorner[kEdge[e][0]][q] + kCorner[kEdge[e][1]][q]);
}
// z-component of cross(q - p, t - p) projected on the normal
double side(const double p[3], const double q[3], const int t[3], const int n[3]) {
    double a[3] = {q[0] - p[0], q[1] - p[1], q[2] - p[2]};
    double b[3] = {t[0] - p[0], t[1] - p[1], t[2] - p[2]};
    double c[3] = {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
    return c[0] * n[0] + c[1] * n[1] + c[2] * n[2];
}

struct Tables {
    int32_t numVerts[256];
    int32_t tri[256][16];
    int32_t edge[256];
    Tables() {
        for (int c = 0; c < 256; c++) build(c);
    }
    void build(int c) {
        auto set = [&](int v) { return (c >> v) & 1; };
        const bool isolate_set = true;
        int emask = 0;
        for (int e = 0; e < 12; e++) if (set(kEdge[e][0]) != set(kEdge[e][1])) emask |= 1 << e;
        edge[c] = emask;
        int next[12];
        for (int e = 0; e < 12; e++) next[e] = -1;
        for (int f = 0; f < 6; f++) {
            const int* C = kFace[f];
            int fe[4];
            for (int q = 0; q < 4; q++) fe[q] = edge_of(C[q], C[(q + 1) % 4]);
            int ncross = 0;
            for (int q = 0; q < 4; q++) ncross += (emask >> fe[q]) & 1;
            // each segment: edges (ea, eb) and the corner it cuts off
            std::vector<std::pair<std::pair<int, int>, int>> segs;
            if (ncross == 2) {
                int ea = -1, eb = -1;
                for (int q = 0; q < 4; q++) if ((emask >> fe[q]) & 1) { if (ea < 0) ea = fe[q]; else eb = fe[q]; }
                int sc = -1;
                for (int q = 0; q < 4; q++) if (set(C[q])) { sc = C[q]; break; }
                segs.push_back({{ea, eb}, sc});
            } else if (ncross == 4) {
                for (int q = 0; q < 4; q++) {
                    int corner = C[q];
                    if ((bool)set(corner) != isolate_set) continue;
                    int ea = fe[(q + 3) % 4], eb = fe[q];   // the two edges at this corner
                    segs.push_back({{ea, eb}, corner});
                }
            }
            for (auto& s : segs) {
                int ea = s.first.first, eb = s.first.second, x = s.second;
                double P[3], Q[3];
                mid(ea, P); mid(eb, Q);
                double sd = side(P, Q, kCorner[x], kNormal[f]);
                bool want_left = set(x);   // the set side must be on the left
                bool is_left = sd > 0;
                if (is_left != want_left) std::swap(ea, eb);
                next[ea] = eb;
            }
        }
        std::memset(tri[c], 0xff, sizeof(tri[c]));
        for (int q = 0; q < 16; q++) tri[c][q] = 255;
        int nt = 0;
        int visited = 0;
        for (int e0 = 0; e0 < 12; e0++) {
            if (!((emask >> e0) & 1) || ((visited >> e0) & 1)) continue;
            std::vector<int> loop;
            int e = e0;
            while (!((visited >> e) & 1)) { visited |= 1 << e; loop.push_back(e); e = next[e]; if (e < 0) break; }
            for (size_t q = 1; q + 1 < loop.size(); q++) {
                if (nt < 5) {
                    tri[c][3 * nt] = loop[0]; tri[c][3 * nt + 1] = loop[q]; tri[c][3 * nt + 2] = loop[q + 1];
                }
                nt++;
            }
        }
        numVerts[c] = 3 * std::min(nt, 5);
    }
};

const Tables& tables() {
    static Tables t;
    return t;
}

}  // namespace

// exported to the C ABI through capi.cu
extern "C" void mp_internal_mc_tables(int32_t* nv, int32_t* tri, int32_t* edge) {
    const Tables& t = tables();
    if (nv) std::memcpy(nv, t.numVerts, sizeof(t.numVerts));
    if (tri) std::memcpy(tri, t.tri, sizeof(t.tri));
    if (edge) std::memcpy(edge, t.edge, sizeof(t.edge));
}
