// mf_plan.h -- symbolic analysis of the nested-dissection multifrontal LU.
//
// Host-only C++ (no CUDA), shared by the device solver (mfront.cu) and the
// CPU check of the analysis in the test suite.
//
// The three linear systems of a timestep live on the (Ny1, Nx1) P-node grid
// with d unknowns per node (d = 6 for Stokes-Darcy: vx, vy, P, qx, qy, Pf;
// d = 1 for heat and gravity), unknown index = node * d + dof with nodes
// column-major (node = j * Ny1 + i), as in the reference's assembly
// (E:3089-3572, E:4526-4611, E:2798-2848).  Every equation couples a node
// only with the 3 x 3 block of nodes around it, so a line of nodes one node
// wide separates the grid.  The analysis bisects the node rectangle
// recursively (the longer side first) down to leaves of at most `leaf`
// nodes.  Each tree node (front) eliminates its separator (a leaf: its whole
// region) and carries as update unknowns the ring of nodes around its
// region, which lie on separators of its ancestors.  In that order the LU
// needs no pivoting for these row-scaled systems (the residual of one solve
// is 2e-10 relative; one refinement step reaches 2e-14).
//
// Front storage: an M x M dense matrix in 64 x 64 tiles, tile (I, J) at
// off + (J * Mt + I) * 4096 doubles, column-major inside the tile.  Local
// unknowns: [0, k) eliminated, [k, Kp) padding eliminated as identity rows,
// [Kp, Kp + u) update unknowns, [Kp + u, M) zero padding; Kp and M - Kp are
// multiples of 64.
#pragma once
#include <algorithm>
#include <cstdint>
#include <vector>

namespace erebus {

constexpr int MF_TILE = 64;

struct MfFront {
    long long off;       // storage offset (doubles)
    long long var_off;   // offset into vars (M entries)
    long long map_off;   // offset into eamap (2 M entries)
    long long vec_off;   // offset into the front vectors (M doubles)
    int M, Kp, k, u;     // sizes, see above
    int Kt, Mt;          // Kp / 64, M / 64
    int parent, c0, c1;  // front indices (-1: none)
    int level;           // depth in the tree (root 0)
    long long poff;      // offset of the solve's partial sums (-1: none; set by the solver)
};

struct MfPlan {
    int d = 0, ny = 0, nx = 0, leaf = 0;
    long long n = 0;                   // unknowns
    std::vector<MfFront> fronts;       // deepest level first
    std::vector<int> level_begin;      // processing level p: [level_begin[p], level_begin[p+1])
    std::vector<int> vars;             // per front, M local -> global unknown (-1 padding)
    std::vector<int> eamap;            // per front, 2 M: local -> child update index (-1 none)
    std::vector<long long> elim_pos;   // global unknown -> elimination position
    std::vector<int> owner;            // global unknown -> front that eliminates it
    long long storage = 0;             // doubles of front storage
    long long vec = 0;                 // doubles of front vectors
    int max_kt = 0, max_mt = 0;
};

namespace mfdetail {
struct Region {
    int i0, i1, j0, j1;
};
struct Node {
    Region r;
    bool leaf;
    int sep_axis, sep;        // 0: column j = sep; 1: row i = sep
    int child[2];
    int depth;
};
inline int pad64(int x) { return (x + MF_TILE - 1) / MF_TILE * MF_TILE; }
}  // namespace mfdetail

// Builds the tree and the per-front unknown lists.  Returns false when the
// grid is empty.
inline bool mf_analyse(MfPlan &P, int d, int ny, int nx, int leaf) {
    using namespace mfdetail;
    P = MfPlan();
    P.d = d;
    P.ny = ny;
    P.nx = nx;
    P.leaf = leaf;
    P.n = (long long)d * ny * nx;
    if (ny <= 0 || nx <= 0 || d <= 0) return false;
    std::vector<Node> T;
    // recursive bisection (explicit stack; children pushed before parents
    // are finished so the tree is built top-down)
    struct Item {
        Region r;
        int parent, slot, depth;
    };
    std::vector<Item> stack{{{0, ny, 0, nx}, -1, 0, 0}};
    int root = -1;
    while (!stack.empty()) {
        Item it = stack.back();
        stack.pop_back();
        Region r = it.r;
        int h = r.i1 - r.i0, w = r.j1 - r.j0;
        if (h <= 0 || w <= 0) continue;
        Node nd;
        nd.r = r;
        nd.depth = it.depth;
        nd.child[0] = nd.child[1] = -1;
        nd.leaf = (long long)h * w <= leaf;
        nd.sep_axis = 0;
        nd.sep = 0;
        int id = (int)T.size();
        if (!nd.leaf) {
            if (w >= h) {
                nd.sep_axis = 0;
                nd.sep = (r.j0 + r.j1) / 2;
            } else {
                nd.sep_axis = 1;
                nd.sep = (r.i0 + r.i1) / 2;
            }
        }
        T.push_back(nd);
        if (it.parent >= 0) T[it.parent].child[it.slot] = id;
        else root = id;
        if (!nd.leaf) {
            Region a = r, b = r;
            if (nd.sep_axis == 0) {
                a.j1 = nd.sep;
                b.j0 = nd.sep + 1;
            } else {
                a.i1 = nd.sep;
                b.i0 = nd.sep + 1;
            }
            stack.push_back({b, id, 1, it.depth + 1});
            stack.push_back({a, id, 0, it.depth + 1});
        }
    }
    if (root < 0) return false;
    // a separator that split off an empty side leaves one child; keep the
    // child in slot 0
    for (Node &nd : T)
        if (nd.child[0] < 0 && nd.child[1] >= 0) std::swap(nd.child[0], nd.child[1]);
    int maxdepth = 0;
    for (const Node &nd : T) maxdepth = std::max(maxdepth, nd.depth);
    // front order: deepest level first, tree order inside a level
    std::vector<int> order;
    P.level_begin.clear();
    for (int dep = maxdepth; dep >= 0; dep--) {
        P.level_begin.push_back((int)order.size());
        for (int t = 0; t < (int)T.size(); t++)
            if (T[t].depth == dep) order.push_back(t);
    }
    P.level_begin.push_back((int)order.size());
    std::vector<int> front_of_node(T.size());
    for (int f = 0; f < (int)order.size(); f++) front_of_node[order[f]] = f;
    // unknown lists
    P.fronts.resize(order.size());
    P.elim_pos.assign(P.n, -1);
    P.owner.assign(P.n, -1);
    long long pos = 0, off = 0, voff = 0, vec = 0;
    auto node_id = [&](int i, int j) { return (long long)j * ny + i; };
    for (int f = 0; f < (int)order.size(); f++) {
        const Node &nd = T[order[f]];
        std::vector<long long> elim, ring;
        const Region &r = nd.r;
        if (nd.leaf) {
            for (int j = r.j0; j < r.j1; j++)
                for (int i = r.i0; i < r.i1; i++) elim.push_back(node_id(i, j));
        } else if (nd.sep_axis == 0) {
            for (int i = r.i0; i < r.i1; i++) elim.push_back(node_id(i, nd.sep));
        } else {
            for (int j = r.j0; j < r.j1; j++) elim.push_back(node_id(nd.sep, j));
        }
        int bi0 = std::max(r.i0 - 1, 0), bi1 = std::min(r.i1 + 1, ny);
        int bj0 = std::max(r.j0 - 1, 0), bj1 = std::min(r.j1 + 1, nx);
        for (int j = bj0; j < bj1; j++)
            for (int i = bi0; i < bi1; i++)
                if (i < r.i0 || i >= r.i1 || j < r.j0 || j >= r.j1) ring.push_back(node_id(i, j));
        MfFront &F = P.fronts[f];
        F.k = (int)elim.size() * d;
        F.u = (int)ring.size() * d;
        F.Kp = pad64(F.k);
        F.M = F.Kp + pad64(F.u);
        F.Kt = F.Kp / MF_TILE;
        F.Mt = F.M / MF_TILE;
        F.level = nd.depth;
        F.poff = -1;
        F.off = off;
        F.var_off = voff;
        F.map_off = 2 * voff;
        F.vec_off = vec;
        off += (long long)F.M * F.M;
        voff += F.M;
        vec += F.M;
        F.c0 = nd.child[0] >= 0 ? front_of_node[nd.child[0]] : -1;
        F.c1 = nd.child[1] >= 0 ? front_of_node[nd.child[1]] : -1;
        F.parent = -1;
        P.vars.resize(voff, -1);
        int *v = &P.vars[F.var_off];
        int a = 0;
        for (long long nn : elim)
            for (int t = 0; t < d; t++) {
                long long g = nn * d + t;
                v[a++] = (int)g;
                P.elim_pos[g] = pos++;
                P.owner[g] = f;
            }
        a = F.Kp;
        for (long long nn : ring)
            for (int t = 0; t < d; t++) v[a++] = (int)(nn * d + t);
        P.max_kt = std::max(P.max_kt, F.Kt);
        P.max_mt = std::max(P.max_mt, F.Mt);
    }
    for (int f = 0; f < (int)P.fronts.size(); f++) {
        if (P.fronts[f].c0 >= 0) P.fronts[P.fronts[f].c0].parent = f;
        if (P.fronts[f].c1 >= 0) P.fronts[P.fronts[f].c1].parent = f;
    }
    P.storage = off;
    P.vec = vec;
    // extend-add maps: local index of the parent -> update index in a child
    P.eamap.assign(2 * voff, -1);
    std::vector<int> loc(P.n, -1);
    for (int f = 0; f < (int)P.fronts.size(); f++) {
        const MfFront &F = P.fronts[f];
        for (int s = 0; s < 2; s++) {
            int c = s == 0 ? F.c0 : F.c1;
            if (c < 0) continue;
            const MfFront &C = P.fronts[c];
            const int *cv = &P.vars[C.var_off];
            for (int a = C.Kp; a < C.Kp + C.u; a++) loc[cv[a]] = a - C.Kp;
            const int *fv = &P.vars[F.var_off];
            for (int a = 0; a < F.M; a++)
                if (fv[a] >= 0) P.eamap[F.map_off + 2 * a + s] = loc[fv[a]];
            for (int a = C.Kp; a < C.Kp + C.u; a++) loc[cv[a]] = -1;
        }
    }
    for (long long g = 0; g < P.n; g++)
        if (P.elim_pos[g] < 0) return false;
    return true;
}

// Storage offset of local element (a, b) of front F.
inline long long mf_elem(const MfFront &F, int a, int b) {
    return F.off + ((long long)(b / MF_TILE) * F.Mt + a / MF_TILE) * MF_TILE * MF_TILE +
           (long long)(b % MF_TILE) * MF_TILE + a % MF_TILE;
}

// Targets of the assembled entries: for ELL entry e = row * ell + slot with
// column c >= 0 and row < n, the storage offset in the front that
// eliminates the first of (row, c); -1 otherwise.  Returns false if an entry
// couples unknowns that no front holds together (a pattern the analysis
// does not cover).
inline bool mf_targets(const MfPlan &P, const int *ell_cols, long long rows, int ell,
                       std::vector<long long> &target) {
    target.assign(rows * ell, -1);
    // group entries by owning front
    std::vector<long long> cnt(P.fronts.size() + 1, 0);
    std::vector<int> ownf(rows * ell, -1);
    for (long long r = 0; r < rows && r < P.n; r++)
        for (int s = 0; s < ell; s++) {
            int c = ell_cols[r * ell + s];
            if (c < 0) continue;
            if (c >= P.n) return false;
            long long first = P.elim_pos[r] <= P.elim_pos[c] ? r : c;
            int f = P.owner[first];
            ownf[r * ell + s] = f;
            cnt[f + 1]++;
        }
    for (size_t f = 0; f < P.fronts.size(); f++) cnt[f + 1] += cnt[f];
    std::vector<long long> ent(cnt.back());
    std::vector<long long> fill(cnt.begin(), cnt.end() - 1);
    for (long long e = 0; e < rows * ell; e++)
        if (ownf[e] >= 0) ent[fill[ownf[e]]++] = e;
    std::vector<int> loc(P.n, -1);
    for (size_t f = 0; f < P.fronts.size(); f++) {
        const MfFront &F = P.fronts[f];
        const int *v = &P.vars[F.var_off];
        for (int a = 0; a < F.M; a++)
            if (v[a] >= 0) loc[v[a]] = a;
        for (long long q = cnt[f]; q < cnt[f + 1]; q++) {
            long long e = ent[q];
            long long r = e / ell;
            int c = ell_cols[e];
            int lr = loc[r], lc = loc[c];
            if (lr < 0 || lc < 0) return false;
            target[e] = mf_elem(F, lr, lc);
        }
        for (int a = 0; a < F.M; a++)
            if (v[a] >= 0) loc[v[a]] = -1;
    }
    return true;
}

}  // namespace erebus
