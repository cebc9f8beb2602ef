// CPU oracle for the grid-kNN -> EGT -> Taubin -> normals path.
//
// ORACLE / TEST INFRASTRUCTURE.  This is a plain C++17/OpenMP restatement of the
// reference implementation (agalex1974/MultiGPUEGTSmoothing) used only by the
// tests, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, as the
// checker.  The product never links it.  Every function cites the reference
// file:line it follows.  Parity of this oracle with the reference itself is
// pinned by the golden fixtures in tests/golden (generated by running the
// unmodified reference, see tests/golden/make_golden.py).
//
// Conventions (all arrays are caller-owned):
//   xyz        original points, AoS float32 [n*3]
//   pos        normalised points in cell-sorted order, SoA float32 [3*n]
//   perm       sorted slot -> original index, int32 [n]
//   lists      sorted-space neighbour lists, int32 [n*k], -1 padded
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <queue>
#include <set>
#include <unordered_set>
#include <vector>
#include <omp.h>

#include "fp_shapes.h"

using namespace fpshape;

namespace {

constexpr float kEps = 1e-6f;          // GridStructure eps (main.cpp:108)
constexpr int kBuckets = 1024;         // level-0 bucket count (main.cpp:108)
constexpr int kMaxPointsInCube = 100000;  // MAX_PNTS_IN_CUBE default (GridKNNCuda.cu:652)
constexpr int kLevels = 8;             // levels 0..7 (B = 1024..8) are searched

// Reference GridKNNCuda.cu:1042-1071 (InitStructure): one scalar cube for all axes.
void cube_extents(const float* xyz, int n, float& mn, float& mx) {
    float lo[3] = {1e8f, 1e8f, 1e8f}, hi[3] = {-1e8f, -1e8f, -1e8f};
    for (int i = 0; i < n; i++)
        for (int d = 0; d < 3; d++) {
            lo[d] = std::min(lo[d], xyz[3 * (size_t)i + d]);
            hi[d] = std::max(hi[d], xyz[3 * (size_t)i + d]);
        }
    for (int d = 0; d < 3; d++) { lo[d] = lo[d] - 1e-6f; hi[d] = hi[d] + 1e-6f; }
    mn = std::min(std::min(lo[0], lo[1]), lo[2]);
    mx = std::max(std::max(hi[0], hi[1]), hi[2]);
}

// Cell coordinate (GridKNNCuda.cu:74-88, :649-653): (int)((x-a)/(b-a)*B).
inline int cell_coord(float x, float a, float b, int B) {
    return (int)((x - a) / (b - a) * (float)B);
}

struct Grid {
    int n = 0;
    float mn = 0, mx = 0;          // normalisation cube
    float a = -kEps, b = 0;        // unit-cube bounds with eps
    std::vector<int> perm;         // sorted slot -> original
    std::vector<float> x, y, z;    // normalised, sorted
    std::vector<int> cx, cy, cz;   // level-0 cell coords per sorted point
    struct Level {
        int B = 0;
        std::vector<int> keys;     // unique occupied cell keys, ascending
        std::vector<int> start;    // start offset of each cell in `order`
        std::vector<int> order;    // sorted indices grouped by cell, ascending inside a cell
    } lv[kLevels];
};

// InitStructure (GridKNNCuda.cu:1023-1133): normalise, level-0 key, stable sort, gather.
void build_grid(const float* xyz, int n, Grid& g, int levels) {
    g.n = n;
    cube_extents(xyz, n, g.mn, g.mx);
    g.b = (float)(1.0 + (double)kEps);
    const float d = g.mx - g.mn;
    std::vector<float> nx(n), ny(n), nz(n);
    std::vector<int> key(n);
    for (int i = 0; i < n; i++) {
        nx[i] = (xyz[3 * (size_t)i] - g.mn) / d;
        ny[i] = (xyz[3 * (size_t)i + 1] - g.mn) / d;
        nz[i] = (xyz[3 * (size_t)i + 2] - g.mn) / d;
        int xi = cell_coord(nx[i], g.a, g.b, kBuckets);
        int yi = cell_coord(ny[i], g.a, g.b, kBuckets);
        int zi = cell_coord(nz[i], g.a, g.b, kBuckets);
        key[i] = xi + yi * kBuckets + zi * kBuckets * kBuckets;
    }
    g.perm.resize(n);
    std::iota(g.perm.begin(), g.perm.end(), 0);
    std::stable_sort(g.perm.begin(), g.perm.end(), [&](int p, int q) { return key[p] < key[q]; });
    g.x.resize(n); g.y.resize(n); g.z.resize(n);
    g.cx.resize(n); g.cy.resize(n); g.cz.resize(n);
    for (int s = 0; s < n; s++) {
        int o = g.perm[s];
        g.x[s] = nx[o]; g.y[s] = ny[o]; g.z[s] = nz[o];
        g.cx[s] = cell_coord(g.x[s], g.a, g.b, kBuckets);
        g.cy[s] = cell_coord(g.y[s], g.a, g.b, kBuckets);
        g.cz[s] = cell_coord(g.z[s], g.a, g.b, kBuckets);
    }
    // Levels (getBuckets / InitializeLevel, GridKNNCuda.cu:898-946): a stable sort
    // of the sorted indices by the level-L key.  Level-L cell = level-0 cell >> L
    // because u*B_L = (u*1024)/2^L exactly in floating point.
    for (int L = 0; L < levels; L++) {
        auto& lv = g.lv[L];
        lv.B = kBuckets >> L;
        std::vector<int> kL(n);
        for (int s = 0; s < n; s++)
            kL[s] = (g.cx[s] >> L) + (g.cy[s] >> L) * lv.B + (g.cz[s] >> L) * lv.B * lv.B;
        lv.order.resize(n);
        std::iota(lv.order.begin(), lv.order.end(), 0);
        std::stable_sort(lv.order.begin(), lv.order.end(), [&](int p, int q) { return kL[p] < kL[q]; });
        lv.keys.clear(); lv.start.clear();
        for (int i = 0; i < n; i++) {
            int kk = kL[lv.order[i]];
            if (i == 0 || kk != lv.keys.back()) { lv.keys.push_back(kk); lv.start.push_back(i); }
        }
        lv.start.push_back(n);
    }
}

// FindPosition (GridKNNCuda.cu:126-143): binary search that returns the slot of
// an equal element if one is hit, otherwise the insertion point.
inline int find_position(const float* a, float x, int low, int high) {
    while (low <= high) {
        int mid = low + (high - low) / 2;
        if (a[mid] == x) return mid;
        if (a[mid] < x) low = mid + 1;
        else high = mid - 1;
    }
    return low + (high - low) / 2;
}

// newNeighborSearch::appendDistanceGrid (GridKNNCuda.cu:311-339).
inline void append(float* dist, int* idx, int k, int& counter, float d, int p) {
    if (!(d < dist[k - 1])) return;
    for (int i = 0; i < counter; i++)
        if (idx[i] == p) return;
    int pos = find_position(dist, d, 0, counter - 1);
    if (counter == k) counter--;
    for (int i = counter - 1; i >= pos; i--) { dist[i + 1] = dist[i]; idx[i + 1] = idx[i]; }
    dist[pos] = d; idx[pos] = p;
    counter++;
}

// Shell cell order of GRIDCUDAKNNSELF_COMPACT for offset 1 (GridKNNCuda.cu:2480-2551).
const int kShell[26][3] = {
    {0, 0, -1}, {0, 0, 1},
    {0, -1, 0}, {0, 1, 0},
    {-1, 0, 0}, {1, 0, 0},
    {-1, -1, 0}, {-1, 1, 0}, {1, -1, 0}, {1, 1, 0},
    {-1, 0, -1}, {-1, 0, 1}, {1, 0, -1}, {1, 0, 1},
    {0, -1, -1}, {0, -1, 1}, {0, 1, -1}, {0, 1, 1},
    {-1, -1, -1}, {-1, -1, 1}, {-1, 1, -1}, {-1, 1, 1}, {1, -1, -1}, {1, -1, 1}, {1, 1, -1}, {1, 1, 1},
};

struct KnnStats { long long visited_points = 0; int max_level = 0; };

// Continue decision on the last cube of a shell (GridKNNCuda.cu:694-741) for a
// query whose list holds `counter` entries with k-th distance `kth`: true =
// search the next shell.
bool decide_more(const Grid& g, int q, int L, int o, int counter, int k, float kth, float thres) {
    const int B = g.lv[L].B;
    const float h = (g.b - g.a) / (float)B;
    const int ci[3] = {g.cx[q] >> L, g.cy[q] >> L, g.cz[q] >> L};
    const float c[3] = {g.x[q], g.y[q], g.z[q]};
    const float xmin = g.a;
    if (counter < k) {
        const float st = std::sqrt(thres);
        for (int d = 0; d < 3; d++) {
            if (ci[d] - o >= 0 && st > face_lo(c[d], xmin, (float)(ci[d] - o), h)) return true;
            if (ci[d] + o + 1 <= B && st > face_hi(c[d], xmin, (float)(ci[d] + o + 1), h)) return true;
        }
        return false;
    }
    const float r = std::sqrt(kth);
    bool more = false;
    for (int d = 0; d < 3; d++) {
        if (ci[d] - o >= 0 && r >= face_lo(c[d], xmin, (float)(ci[d] - o), h)) more = true;
        if (ci[d] + o + 1 <= B && r >= face_hi(c[d], xmin, (float)(ci[d] + o + 1), h)) more = true;
    }
    return more;
}

// One query of GRIDCUDAKNNSELF_COMPACT (GridKNNCuda.cu:2322-2586) with the
// kernel body construct_neighbors_self_compact (GridKNNCuda.cu:647-743).
// Returns the level reached (0..7, or 8 when the query ran out of levels).
int knn_query(const Grid& g, int q, int k, float thres, float* dist, int* idx, int& counter,
              bool& invalid, long long& visited) {
    for (int i = 0; i < k; i++) { dist[i] = 1e10f; idx[i] = -1; }
    counter = 0;
    invalid = false;
    const float xq = g.x[q], yq = g.y[q], zq = g.z[q];

    auto visit = [&](int L, int cx, int cy, int cz) {
        const auto& lv = g.lv[L];
        if (cx < 0 || cx >= lv.B || cy < 0 || cy >= lv.B || cz < 0 || cz >= lv.B) return;
        int key = cx + cy * lv.B + cz * lv.B * lv.B;
        auto it = std::lower_bound(lv.keys.begin(), lv.keys.end(), key);
        if (it == lv.keys.end() || *it != key) return;
        if (invalid) return;
        size_t c = it - lv.keys.begin();
        int s0 = lv.start[c], s1 = lv.start[c + 1];
        if (s1 - s0 >= kMaxPointsInCube) { invalid = true; return; }
        for (int j = s0; j < s1; j++) {
            int p = lv.order[j];
            if (p == q) continue;
            float d = dist3(xq, yq, zq, g.x[p], g.y[p], g.z[p]);
            visited++;
            if (d <= thres) append(dist, idx, k, counter, d, p);
        }
    };
    auto decide = [&](int L, int o) -> bool {
        if (invalid) return false;
        return decide_more(g, q, L, o, counter, k, dist[k - 1], thres);
    };

    visit(0, g.cx[q], g.cy[q], g.cz[q]);
    bool cont = decide(0, 0);
    int L = 0;
    int reached = 0;
    while (cont) {
        reached = L;
        const int xi = g.cx[q] >> L, yi = g.cy[q] >> L, zi = g.cz[q] >> L;
        for (int s = 0; s < 26; s++) visit(L, xi + kShell[s][0], yi + kShell[s][1], zi + kShell[s][2]);
        cont = decide(L, 1);
        if (L == kLevels - 1) break;
        L++;
    }
    // A query still searching after the B=8 ring is invalid (GridKNNCuda.cu:2572-2586).
    if (cont) { invalid = true; reached = kLevels; }
    if (invalid)
        for (int i = 0; i < k; i++) idx[i] = -1;
    return reached;
}

// ---------------------------------------------------------------------------
// Query-vs-reference kNN: GridStructure::GRIDCUDAKNNCompact (GridKNNCuda.cu:
// 1645-1939) with its kernel construct_neighbors (GridKNNCuda.cu:340-438).
// The same level/shell schedule as the self search (own level-0 cell, then the
// 26-cell shell at levels 0..7, a query still searching after B = 8 is
// invalid), with these differences, each from the cited lines:
//   * the query points are normalised with the reference cloud's cube
//     (normalize_points, :841-849; :1700-1706) and may lie outside it;
//   * the query's cell at each level is computed from its coordinate,
//     (int)((x - a)/(b - a) * B_L) (:349-351), which truncates toward zero
//     for coordinates below the cube;
//   * no point is excluded as "self" (:357-365);
//   * admission is dist < thres (:363), strict;
//   * with fewer than k neighbours the search continues when
//     sqrt(thres) >= a face distance (:377-392), otherwise when
//     sqrt(k-th) >= a face distance (:393-420);
//   * cells outside the grid are skipped, never invalidating (:352-354, :370-374);
//   * an oversized cell invalidates the query (:367-369).
// lists: [k] reference sorted-space ids of query (x, y, z), normalised.
struct QueryCells { int c[kLevels][3]; };

inline QueryCells query_cells(const Grid& g, float x, float y, float z) {
    QueryCells qc;
    for (int L = 0; L < kLevels; L++) {
        const int B = kBuckets >> L;
        qc.c[L][0] = cell_coord(x, g.a, g.b, B);
        qc.c[L][1] = cell_coord(y, g.a, g.b, B);
        qc.c[L][2] = cell_coord(z, g.a, g.b, B);
    }
    return qc;
}

bool decide_more_query(const Grid& g, const QueryCells& qc, float x, float y, float z, int L, int o, int counter,
                       int k, float kth, float thres) {
    const int B = g.lv[L].B;
    const float h = (g.b - g.a) / (float)B;
    const float c[3] = {x, y, z};
    const float xmin = g.a;
    const float r = counter < k ? std::sqrt(thres) : std::sqrt(kth);
    for (int d = 0; d < 3; d++) {
        const int ci = qc.c[L][d];
        if (ci - o >= 0 && r >= face_lo(c[d], xmin, (float)(ci - o), h)) return true;
        if (ci + o + 1 <= B && r >= face_hi(c[d], xmin, (float)(ci + o + 1), h)) return true;
    }
    return false;
}

int knn_foreign_query(const Grid& g, float xq, float yq, float zq, int k, float thres, float* dist, int* idx,
                      int& counter, bool& invalid) {
    for (int i = 0; i < k; i++) { dist[i] = 1e10f; idx[i] = -1; }
    counter = 0;
    invalid = false;
    const QueryCells qc = query_cells(g, xq, yq, zq);
    auto visit = [&](int L, int cx, int cy, int cz) {
        const auto& lv = g.lv[L];
        if (cx < 0 || cx >= lv.B || cy < 0 || cy >= lv.B || cz < 0 || cz >= lv.B) return;
        const int key = cx + cy * lv.B + cz * lv.B * lv.B;
        auto it = std::lower_bound(lv.keys.begin(), lv.keys.end(), key);
        if (it == lv.keys.end() || *it != key) return;
        if (invalid) return;
        const size_t c = it - lv.keys.begin();
        const int s0 = lv.start[c], s1 = lv.start[c + 1];
        if (s1 - s0 >= kMaxPointsInCube) { invalid = true; return; }
        for (int j = s0; j < s1; j++) {
            const int p = lv.order[j];
            const float d = dist3(xq, yq, zq, g.x[p], g.y[p], g.z[p]);
            if (d < thres) append(dist, idx, k, counter, d, p);
        }
    };
    auto decide = [&](int L, int o) -> bool {
        if (invalid) return false;
        return decide_more_query(g, qc, xq, yq, zq, L, o, counter, k, dist[k - 1], thres);
    };
    visit(0, qc.c[0][0], qc.c[0][1], qc.c[0][2]);
    bool cont = decide(0, 0);
    int L = 0, reached = 0;
    while (cont) {
        reached = L;
        for (int s = 0; s < 26; s++)
            visit(L, qc.c[L][0] + kShell[s][0], qc.c[L][1] + kShell[s][1], qc.c[L][2] + kShell[s][2]);
        cont = decide(L, 1);
        if (L == kLevels - 1) break;
        L++;
    }
    if (cont) { invalid = true; reached = kLevels; }  // GridKNNCuda.cu:1921-1928
    if (invalid)
        for (int i = 0; i < k; i++) idx[i] = -1;
    return reached;
}

// ---------------------------------------------------------------------------
// Learned search proposal (an extension of this project; the reference has no
// counterpart).  A proposal class names a box of level-L cells of half-width R
// around the query's level-L cell; the last class means "run the plain search".
// The box search keeps the k+1 smallest distances of the box and is accepted
// only when it provably equals the plain search's list:
//   (1) at least k candidates, and the k+1 smallest distances pairwise distinct
//       (then any candidate order yields the same sorted list);
//   (2) the k-th distance ball lies inside the box with a margin of 2e-6 in
//       normalised units (all points outside the box are strictly farther), so
//       the k smallest of the box are the k smallest of the cloud, G;
//   (3) the plain search's stop step is replayed: for step s (own cell, then
//       the ring at level s-1) the plain list equals G once the visited block
//       holds G, so the decision there is decide_more(kth(G)); before that the
//       plain k-th distance is >= kth(G) and the search continues whenever
//       decide_more(kth(G)) and the under-full branch both say "continue";
//   (4) no cell of a level the plain search visits holds >= MAX_PNTS_IN_CUBE
//       points (the plain search would have marked the query invalid).
// Any failed check falls back to the plain search.
struct BoxClass { int level, radius; };
constexpr int kProposalClasses = 16;
const BoxClass kBox[kProposalClasses - 1] = {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 5}, {0, 6}, {1, 4}, {1, 5},
                                             {1, 6}, {2, 4}, {2, 5}, {2, 6}, {3, 4}, {3, 5}, {3, 6}};
constexpr double kBoxMargin = 2e-6;

// points in cells [x0, x1] of row (cy, cz) at level L (clipped to the grid)
int row_count(const Grid& g, int L, int x0, int x1, int cy, int cz) {
    const auto& lv = g.lv[L];
    if (cy < 0 || cy >= lv.B || cz < 0 || cz >= lv.B) return 0;
    x0 = std::max(x0, 0);
    x1 = std::min(x1, lv.B - 1);
    if (x0 > x1) return 0;
    const int base = cy * lv.B + cz * lv.B * lv.B;
    auto i0 = std::lower_bound(lv.keys.begin(), lv.keys.end(), base + x0) - lv.keys.begin();
    auto i1 = std::lower_bound(lv.keys.begin(), lv.keys.end(), base + x1 + 1) - lv.keys.begin();
    return lv.start[i1] - lv.start[i0];
}

// 8 features: log2(1+count)/16 of the query's own cell at levels 0..5 and of
// its 3x3x3 level-0 block, and twice the smallest fractional distance of the
// query to a face of its level-0 cell.
void proposal_features(const Grid& g, int q, float f[8]) {
    for (int L = 0; L < 6; L++) {
        const int c = row_count(g, L, g.cx[q] >> L, g.cx[q] >> L, g.cy[q] >> L, g.cz[q] >> L);
        f[L] = std::log2(1.0f + (float)c) * 0.0625f;
    }
    int blk = 0;
    for (int dz = -1; dz <= 1; dz++)
        for (int dy = -1; dy <= 1; dy++) blk += row_count(g, 0, g.cx[q] - 1, g.cx[q] + 1, g.cy[q] + dy, g.cz[q] + dz);
    f[6] = std::log2(1.0f + (float)blk) * 0.0625f;
    const float c[3] = {g.x[q], g.y[q], g.z[q]};
    const int ci[3] = {g.cx[q], g.cy[q], g.cz[q]};
    float m = 0.5f;
    for (int d = 0; d < 3; d++) {
        const float v = (c[d] - g.a) / (g.b - g.a) * (float)kBuckets;
        const float fr = v - (float)ci[d];
        m = std::min(m, std::min(fr, 1.0f - fr));
    }
    f[7] = 2.0f * std::max(m, 0.0f);
}

// Level-0 cell range [lo, end) per axis of the box of class `cls` whose
// (y, z) half-width is `ryz` (<= radius) level-L cells.
void box_bounds(const Grid& g, int q, int cls, int ryz, int lo[3], int end[3]) {
    const int L = kBox[cls].level, R = kBox[cls].radius;
    const int ci[3] = {g.cx[q] >> L, g.cy[q] >> L, g.cz[q] >> L};
    for (int d = 0; d < 3; d++) {
        const int r = d == 0 ? R : ryz;
        lo[d] = (ci[d] - r) * (1 << L);
        end[d] = (ci[d] + r + 1) * (1 << L);
    }
}

// Condition (2): the ball of radius sqrt(kth) + margin is inside the box.
bool ball_in_box(const Grid& g, int q, float kth, const int lo[3], const int end[3]) {
    const double r = std::sqrt((double)kth) + kBoxMargin;
    const double h0 = (double)((g.b - g.a) / (float)kBuckets);
    const double c[3] = {g.x[q], g.y[q], g.z[q]};
    for (int d = 0; d < 3; d++) {
        if (lo[d] > 0 && !(r < c[d] - ((double)g.a + lo[d] * h0))) return false;
        if (end[d] < kBuckets && !(r < ((double)g.a + end[d] * h0) - c[d])) return false;
    }
    return true;
}

// First plain-search step (0 = own cell, s = ring at level s-1) at which p is visited.
int visit_step(const Grid& g, int q, int p) {
    if (g.cx[p] == g.cx[q] && g.cy[p] == g.cy[q] && g.cz[p] == g.cz[q]) return 0;
    for (int L = 0; L < kLevels; L++) {
        if (std::abs((g.cx[p] >> L) - (g.cx[q] >> L)) <= 1 && std::abs((g.cy[p] >> L) - (g.cy[q] >> L)) <= 1 &&
            std::abs((g.cz[p] >> L) - (g.cz[q] >> L)) <= 1)
            return L + 1;
    }
    return kLevels + 1;
}

// Label of a query from the plain search's k-th distance: the cheapest class
// whose box passes condition (2), else the plain class.
int proposal_label(const Grid& g, int q, int counter, int k, float kth) {
    if (counter < k) return kProposalClasses - 1;
    for (int c = 0; c < kProposalClasses - 1; c++) {
        int lo[3], end[3];
        box_bounds(g, q, c, kBox[c].radius, lo, end);
        if (ball_in_box(g, q, kth, lo, end)) return c;
    }
    return kProposalClasses - 1;
}

// Box search + certification for one query.  Returns true (and fills
// idx[0..k), reached) when the box result is certified equal to the plain
// search's; `visited` counts the candidates examined.
bool box_query(const Grid& g, int q, int k, int cls, float thres, const int* maxpop, int* idx, int& reached,
               long long& visited, std::vector<std::pair<float, int>>& cand) {
    const int L = kBox[cls].level, R = kBox[cls].radius;
    const auto& lv = g.lv[L];
    const int ci[3] = {g.cx[q] >> L, g.cy[q] >> L, g.cz[q] >> L};
    cand.clear();
    for (int dz = -R; dz <= R; dz++)
        for (int dy = -R; dy <= R; dy++) {
            const int cy = ci[1] + dy, cz = ci[2] + dz;
            if (cy < 0 || cy >= lv.B || cz < 0 || cz >= lv.B) continue;
            const int x0 = std::max(ci[0] - R, 0), x1 = std::min(ci[0] + R, lv.B - 1);
            const int base = cy * lv.B + cz * lv.B * lv.B;
            auto i0 = std::lower_bound(lv.keys.begin(), lv.keys.end(), base + x0) - lv.keys.begin();
            auto i1 = std::lower_bound(lv.keys.begin(), lv.keys.end(), base + x1 + 1) - lv.keys.begin();
            for (int j = lv.start[i0]; j < lv.start[i1]; j++) {
                const int p = lv.order[j];
                if (p == q) continue;
                const float d = dist3(g.x[q], g.y[q], g.z[q], g.x[p], g.y[p], g.z[p]);
                visited++;
                if (d <= thres) cand.push_back({d, p});
            }
        }
    const int m = (int)cand.size();
    if (m < k) return false;
    const int keep = std::min(m, k + 1);
    std::partial_sort(cand.begin(), cand.begin() + keep, cand.end(),
                      [](const std::pair<float, int>& a, const std::pair<float, int>& b) { return a.first < b.first; });
    for (int i = 1; i < keep; i++)                                     // (1)
        if (!(cand[i - 1].first < cand[i].first)) return false;
    const float kth = cand[k - 1].first;
    int lo[3], end[3];
    box_bounds(g, q, cls, R, lo, end);
    if (!ball_in_box(g, q, kth, lo, end)) return false;                // (2)
    int sg = 0;
    for (int i = 0; i < k; i++) sg = std::max(sg, visit_step(g, q, cand[i].second));
    int sf = -1;                                                       // (3)
    for (int s = 0; s <= kLevels; s++) {
        const int Ls = s == 0 ? 0 : s - 1, o = s == 0 ? 0 : 1;
        const bool more = decide_more(g, q, Ls, o, k, k, kth, thres);
        if (!more) { sf = s; break; }
        if (!decide_more(g, q, Ls, o, 0, k, kth, thres)) return false;
    }
    if (sf < 0 || sg > sf) return false;
    for (int l = 0; l <= std::max(sf - 1, 0); l++)                     // (4)
        if (maxpop[l] >= kMaxPointsInCube) return false;
    for (int i = 0; i < k; i++) idx[i] = cand[i].second;
    reached = std::max(sf - 1, 0);
    return true;
}

void level_maxpop(const Grid& g, int* maxpop) {
    for (int L = 0; L < kLevels; L++) {
        int m = 0;
        for (size_t c = 0; c + 1 < g.lv[L].start.size(); c++) m = std::max(m, g.lv[L].start[c + 1] - g.lv[L].start[c]);
        maxpop[L] = m;
    }
}

// EGT predicate isEllipicGabrielNeighbor_GKNN (EGT_CUDA.cu:136-170) with its
// helpers (EGT_CUDA.cu:34-134).
inline void normalize3(float& x, float& y, float& z) {
    float nrm = std::sqrt(sq3(x, y, z));
    x /= nrm; y /= nrm; z /= nrm;
}

bool egt_keep(const float* X, const float* Y, const float* Z, const int* row, int j,
              float x, float y, float z, float alpha) {
    const int nb = row[j];
    float xi = X[nb], yi = Y[nb], zi = Z[nb];
    float xo = 0.5f * (xi + x), yo = 0.5f * (yi + y), zo = 0.5f * (zi + z);
    float d = std::sqrt(dist3(xi, yi, zi, x, y, z)) / 2.0f;
    if ((double)d < 1e-6) return true;
    float ax = xi - x, ay = yi - y, az = zi - z;
    if ((double)std::sqrt(sq3(ax, ay, az)) < 1e-6) return true;
    normalize3(ax, ay, az);
    // perpendicular (EGT_CUDA.cu:61-95)
    float mxv = std::fabs(ax);
    int ci = 0;
    if (mxv < std::fabs(ay)) { ci = 1; mxv = std::fabs(ay); }
    if (mxv < std::fabs(az)) ci = 2;
    float px = 1.0f, py = 1.0f, pz = 1.0f;
    if (ci == 0) px = (-ay * py - az * pz) / ax;
    else if (ci == 1) py = (-ax * px - az * pz) / ay;
    else pz = (-ax * px - ay * py) / az;
    normalize3(px, py, pz);
    // third axis = x-axis cross perpendicular (EGT_CUDA.cu:97-104, 126-127)
    float qx = cross1(ay, pz, py, az);
    float qy = cross1(px, az, ax, pz);
    float qz = cross1(ax, py, px, ay);
    normalize3(qx, qy, qz);
    // translation: A * o with a14 = a24 = a34 = 0 (EGT_CUDA.cu:128-133)
    float tx = affine(ax, ay, az, 0.0f, xo, yo, zo);
    float ty = affine(px, py, pz, 0.0f, xo, yo, zo);
    float tz = affine(qx, qy, qz, 0.0f, xo, yo, zo);
    tx = -tx; ty = -ty; tz = -tz;
    const float aa = alpha * alpha;
    const float dd = d * d;
    for (int jj = 0; jj < j; jj++) {
        int m = row[jj];
        if (m < 0) continue;
        float ux = X[m], uy = Y[m], uz = Z[m];
        float lx = affine(ax, ay, az, tx, ux, uy, uz);
        float ly = affine(px, py, pz, ty, ux, uy, uz);
        float lz = affine(qx, qy, qz, tz, ux, uy, uz);
        if (ellipsoid(lx, ly, lz, aa) < dd) return false;
    }
    return true;
}

// ---------------------------------------------------------------------------
// Symmetric 3x3 eigensolver: the iterative Householder + Givens algorithm of
// D. Eberly ("A Robust Eigensolver for 3x3 Symmetric Matrices", Geometric
// Tools), as used by the reference (EigenSolver.cuh:124-392, sorted by
// SortEigenstuff EigenSolver.cuh:29-122).  T = float mirrors the reference's
// rounding shapes; T = double is the FP64 oracle.
template <typename T> struct Fp;
template <> struct Fp<float> {
    static float lin_add(float c, float a, float s, float b) { return lin2_add(c, a, s, b); }
    static float lin_sub(float s, float a, float c, float b) { return lin2_sub(s, a, c, b); }
    static float hyp2(float u, float v) { return sq2(u, v); }
    static float sqrtv(float v) { return std::sqrt(v); }
    static int alpha() { return 149; }
};
template <> struct Fp<double> {
    static double lin_add(double c, double a, double s, double b) { return c * a + s * b; }
    static double lin_sub(double s, double a, double c, double b) { return s * a - c * b; }
    static double hyp2(double u, double v) { return u * u + v * v; }
    static double sqrtv(double v) { return std::sqrt(v); }
    static int alpha() { return 1074; }
};

template <typename T>
void cos_sin(T u, T v, T& c, T& s) {  // GetCosSin (EigenSolver.cuh:353-373)
    T len = Fp<T>::sqrtv(Fp<T>::hyp2(u, v));
    if (len > T(0)) {
        c = u / len; s = v / len;
        if (c > T(0)) { c = -c; s = -s; }
    } else { c = T(-1); s = T(0); }
}

template <typename T>
bool converged(T d0, T d1, T sd) {  // Converged, aggressive = false (EigenSolver.cuh:375-391)
    T sum = std::fabs(d0) + std::fabs(d1);
    return sum + std::fabs(sd) == sum;
}

template <typename T>
void eigen3(T a00, T a01, T a02, T a11, T a12, T a22, T eval[3], T evec[3][3]) {
    using F = Fp<T>;
    const T half = T(0.5), one = T(1);
    bool isRotation = false;
    T c = 0, s = 0;
    cos_sin<T>(a12, -a02, c, s);
    T term0 = F::lin_add(c, a00, s, a01);
    T term1 = F::lin_add(c, a01, s, a11);
    T term2 = F::lin_sub(s, a00, c, a01);
    T term3 = F::lin_sub(s, a01, c, a11);
    T b00 = F::lin_add(c, term0, s, term1);
    T b01 = F::lin_sub(s, term0, c, term1);
    T b11 = F::lin_sub(s, term2, c, term3);
    T b12 = F::lin_sub(s, a02, c, a12);
    T b22 = a22;
    T Q[3][3] = {{c, s, 0}, {s, -c, 0}, {0, 0, 1}};
    int power = 0;
    T c2 = 0, s2 = 0;
    if (std::fabs(b12) <= std::fabs(b01)) {
        std::frexp(b12, &power);
        int imax = 2 * (power + F::alpha() + 1);
        for (int i = 0; i < imax; ++i) {
            cos_sin<T>(half * (b00 - b11), b01, c2, s2);
            s = F::sqrtv(half * (one - c2));
            c = half * s2 / s;
            for (int r = 0; r < 3; ++r) {
                T t0 = F::lin_add(c, Q[r][0], s, Q[r][1]);
                T t1 = Q[r][2];
                T t2 = F::lin_sub(c, Q[r][1], s, Q[r][0]);
                Q[r][0] = t0; Q[r][1] = t1; Q[r][2] = t2;
            }
            isRotation = !isRotation;
            term0 = F::lin_add(c, b00, s, b01);
            term1 = F::lin_add(c, b01, s, b11);
            term2 = F::lin_sub(s, b00, c, b01);
            term3 = F::lin_sub(s, b01, c, b11);
            b00 = F::lin_add(c, term0, s, term1);
            b01 = s * b12;
            b11 = b22;
            b12 = c * b12;
            b22 = F::lin_sub(s, term2, c, term3);
            if (converged<T>(b00, b11, b01)) {
                cos_sin<T>(half * (b00 - b11), b01, c2, s2);
                s = F::sqrtv(half * (one - c2));
                c = half * s2 / s;
                for (int r = 0; r < 3; ++r) {
                    T t0 = F::lin_add(c, Q[r][0], s, Q[r][1]);
                    T t1 = F::lin_sub(s, Q[r][0], c, Q[r][1]);
                    Q[r][0] = t0; Q[r][1] = t1;
                }
                isRotation = !isRotation;
                term0 = F::lin_add(c, b00, s, b01);
                term1 = F::lin_add(c, b01, s, b11);
                term2 = F::lin_sub(s, b00, c, b01);
                term3 = F::lin_sub(s, b01, c, b11);
                b00 = F::lin_add(c, term0, s, term1);
                b11 = F::lin_sub(s, term2, c, term3);
                break;
            }
        }
    } else {
        std::frexp(b01, &power);
        int imax = 2 * (power + F::alpha() + 1);
        for (int i = 0; i < imax; ++i) {
            cos_sin<T>(half * (b11 - b22), b12, c2, s2);
            s = F::sqrtv(half * (one - c2));
            c = half * s2 / s;
            for (int r = 0; r < 3; ++r) {
                T t0 = F::lin_add(c, Q[r][1], s, Q[r][2]);
                T t1 = Q[r][0];
                T t2 = F::lin_sub(c, Q[r][2], s, Q[r][1]);
                Q[r][0] = t0; Q[r][1] = t1; Q[r][2] = t2;
            }
            isRotation = !isRotation;
            term0 = F::lin_add(c, b11, s, b12);
            term1 = F::lin_add(c, b12, s, b22);
            term2 = F::lin_sub(s, b11, c, b12);
            term3 = F::lin_sub(s, b12, c, b22);
            b22 = F::lin_sub(s, term2, c, term3);
            b12 = -s * b01;
            b11 = b00;
            b01 = c * b01;
            b00 = F::lin_add(c, term0, s, term1);
            if (converged<T>(b11, b22, b12)) {
                cos_sin<T>(half * (b11 - b22), b12, c2, s2);
                s = F::sqrtv(half * (one - c2));
                c = half * s2 / s;
                for (int r = 0; r < 3; ++r) {
                    T t0 = F::lin_add(c, Q[r][1], s, Q[r][2]);
                    T t1 = F::lin_sub(s, Q[r][1], c, Q[r][2]);
                    Q[r][1] = t0; Q[r][2] = t1;
                }
                isRotation = !isRotation;
                term0 = F::lin_add(c, b11, s, b12);
                term1 = F::lin_add(c, b12, s, b22);
                term2 = F::lin_sub(s, b11, c, b12);
                term3 = F::lin_sub(s, b12, c, b22);
                b11 = F::lin_add(c, term0, s, term1);
                b22 = F::lin_sub(s, term2, c, term3);
                break;
            }
        }
    }
    T ev[3] = {b00, b11, b22};
    T vec[3][3];
    for (int r = 0; r < 3; ++r)
        for (int col = 0; col < 3; ++col) vec[r][col] = Q[col][r];
    // SortEigenstuff, sortType = +1 (increasing) and right-handed basis.
    int index[3];
    if (ev[0] < ev[1]) {
        if (ev[2] < ev[0]) { index[0] = 2; index[1] = 0; index[2] = 1; }
        else if (ev[2] < ev[1]) { index[0] = 0; index[1] = 2; index[2] = 1; isRotation = !isRotation; }
        else { index[0] = 0; index[1] = 1; index[2] = 2; }
    } else {
        if (ev[2] < ev[1]) { index[0] = 2; index[1] = 1; index[2] = 0; isRotation = !isRotation; }
        else if (ev[2] < ev[0]) { index[0] = 1; index[1] = 2; index[2] = 0; }
        else { index[0] = 1; index[1] = 0; index[2] = 2; isRotation = !isRotation; }
    }
    for (int j = 0; j < 3; ++j) {
        eval[j] = ev[index[j]];
        for (int col = 0; col < 3; ++col) evec[j][col] = vec[index[j]][col];
    }
    if (!isRotation)
        for (int col = 0; col < 3; ++col) evec[2][col] = -evec[2][col];
}

// calculateNormal (Normal_CUDA.cu:87-144), float or double arithmetic.
template <typename T>
void normal_of(const float* X, const float* Y, const float* Z, const int* row, int k, int i, T out[3]) {
    T sx = X[i], sy = Y[i], sz = Z[i];
    int cnt = 1;
    for (int j = 0; j < k; j++) {
        int m = row[j];
        if (m >= 0) { sx += X[m]; sy += Y[m]; sz += Z[m]; cnt++; }
    }
    T cxm = sx / (T)cnt, cym = sy / (T)cnt, czm = sz / (T)cnt;
    T c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
    for (int j = 0; j < k; j++) {
        int m = row[j];
        if (m < 0) continue;
        T dx = X[m] - cxm, dy = Y[m] - cym, dz = Z[m] - czm;
        if constexpr (sizeof(T) == 4) {
            c00 = cov_acc(c00, dx, dx); c01 = cov_acc(c01, dx, dy); c02 = cov_acc(c02, dx, dz);
            c11 = cov_acc(c11, dy, dy); c12 = cov_acc(c12, dy, dz); c22 = cov_acc(c22, dz, dz);
        } else {
            c00 += dx * dx; c01 += dx * dy; c02 += dx * dz; c11 += dy * dy; c12 += dy * dz; c22 += dz * dz;
        }
    }
    T ev[3], vec[3][3];
    eigen3<T>(c00, c01, c02, c11, c12, c22, ev, vec);
    T nx = vec[0][0], ny = vec[0][1], nz = vec[0][2];
    T nrm;
    if constexpr (sizeof(T) == 4) nrm = std::sqrt(sq3(nx, ny, nz));
    else nrm = std::sqrt(nx * nx + ny * ny + nz * nz);
    out[0] = nx / nrm; out[1] = ny / nrm; out[2] = nz / nrm;
}

struct DSU {
    std::vector<int> p;
    explicit DSU(int n) : p(n) { std::iota(p.begin(), p.end(), 0); }
    int find(int a) { while (p[a] != a) { p[a] = p[p[a]]; a = p[a]; } return a; }
    bool unite(int a, int b) { a = find(a); b = find(b); if (a == b) return false; p[a] = b; return true; }
};

}  // namespace

extern "C" {

int orc_num_threads() { return omp_get_max_threads(); }

// Normalisation cube of InitStructure (GridKNNCuda.cu:1042-1071): ext = {min, max}.
void orc_extents(const float* xyz, int n, float* ext) { cube_extents(xyz, n, ext[0], ext[1]); }

// Grid kNN of the reference (GridStructure + GRIDCUDAKNNSELF_COMPACT).
//   lists [n*k] sorted-space neighbours, pos [3n] SoA sorted normalised,
//   perm [n], ext [2], level [n] (optional): level at which the query stopped
//   (0..7, 8 = ran out of levels), kth [n] (optional): k-th distance (1e10 if < k).
// Returns the number of invalid queries.
int orc_knn(const float* xyz, int n, int k, float thres_in, int* lists, float* pos, int* perm, float* ext,
            int* level, float* kth, long long* visited_total) {
    Grid g;
    build_grid(xyz, n, g, kLevels);
    float thres = thres_in;  // GRIDCUDAKNNSELF_COMPACT(k, thres), GridKNNCuda.cu:2324-2325
    thres /= (g.mx - g.mn);
    thres *= thres;
    int invalid_count = 0;
    long long visited_sum = 0;
#pragma omp parallel reduction(+ : invalid_count, visited_sum)
    {
        std::vector<float> dist(k);
#pragma omp for schedule(dynamic, 256)
        for (int q = 0; q < n; q++) {
            int counter;
            bool invalid;
            long long visited = 0;
            int lv = knn_query(g, q, k, thres, dist.data(), lists + (size_t)q * k, counter, invalid, visited);
            visited_sum += visited;
            if (invalid) invalid_count++;
            if (level) level[q] = lv;
            if (kth) kth[q] = counter == k ? dist[k - 1] : 1e10f;
        }
    }
    for (int s = 0; s < n; s++) {
        pos[s] = g.x[s]; pos[n + s] = g.y[s]; pos[2 * (size_t)n + s] = g.z[s];
        perm[s] = g.perm[s];
    }
    ext[0] = g.mn; ext[1] = g.mx;
    if (visited_total) *visited_total = visited_sum;
    return invalid_count;
}

// Query-vs-reference kNN of the reference (GridStructure(ref) +
// GRIDCUDAKNNCompact(queries, k, thres) + GetKNNIndexes, GridKNNCuda.cu:
// 1645-1968): out [nq*k] original reference ids in original query order, -1
// padded (whole row -1 for an invalid query).  Returns the invalid count.
//   status [nq] (optional): 0 = valid, 1 = a visited cell was oversized,
//   2 = still searching after the B = 8 shell.  The reference decides the
//   status-2 rows from a buffer it re-allocates without clearing
//   (recomputeBuffers, GridKNNCuda.cu:1135-1163, read by
//   invalidateNotFinishedNeighbors at :1921-1928), so for them its output is
//   undefined; this restatement invalidates them all.
int orc_knn_query(const float* xyz, int n, const float* q, int nq, int k, float thres_in, int* out,
                  int* status) {
    Grid g;
    build_grid(xyz, n, g, kLevels);
    float thres = thres_in;
    thres /= (g.mx - g.mn);
    thres *= thres;
    const float d = g.mx - g.mn;
    int invalid_count = 0;
#pragma omp parallel reduction(+ : invalid_count)
    {
        std::vector<float> dist(k);
        std::vector<int> idx(k);
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < nq; i++) {
            const float x = (q[3 * (size_t)i] - g.mn) / d, y = (q[3 * (size_t)i + 1] - g.mn) / d,
                        z = (q[3 * (size_t)i + 2] - g.mn) / d;
            int counter;
            bool invalid;
            const int reached = knn_foreign_query(g, x, y, z, k, thres, dist.data(), idx.data(), counter, invalid);
            if (invalid) invalid_count++;
            if (status) status[i] = !invalid ? 0 : (reached == kLevels ? 2 : 1);
            for (int t = 0; t < k; t++) out[(size_t)i * k + t] = idx[t] >= 0 ? g.perm[idx[t]] : -1;
        }
    }
    return invalid_count;
}

// Learned-proposal training data (extension, no reference counterpart):
// features [n*8] and labels [n] of every query in sorted space, labels from
// the plain search's k-th distance.  Returns the number of plain-class labels.
int orc_proposal_data(const float* xyz, int n, int k, float* feats, uint8_t* labels) {
    Grid g;
    build_grid(xyz, n, g, kLevels);
    float thres = 1e8f;
    thres /= (g.mx - g.mn);
    thres *= thres;
    int plain = 0;
#pragma omp parallel reduction(+ : plain)
    {
        std::vector<float> dist(k);
        std::vector<int> idx(k);
#pragma omp for schedule(dynamic, 256)
        for (int q = 0; q < n; q++) {
            int counter;
            bool invalid;
            long long visited = 0;
            knn_query(g, q, k, thres, dist.data(), idx.data(), counter, invalid, visited);
            proposal_features(g, q, feats + (size_t)q * 8);
            const int lab = invalid ? kProposalClasses - 1 : proposal_label(g, q, counter, k, dist[k - 1]);
            labels[q] = (uint8_t)lab;
            plain += lab == kProposalClasses - 1;
        }
    }
    return plain;
}

// Grid kNN through the proposal: per-query class `cls` [n] (sorted space);
// class kProposalClasses-1 or a failed certification runs the plain search.
// lists [n*k] must equal orc_knn's.  certified [n]: 1 = box result used.
// Returns the number of invalid queries; box_visited/plain_visited count the
// candidates examined by each part.
int orc_knn_proposal(const float* xyz, int n, int k, const uint8_t* cls, int* lists, uint8_t* certified,
                     int* level, long long* box_visited, long long* plain_visited) {
    Grid g;
    build_grid(xyz, n, g, kLevels);
    float thres = 1e8f;
    thres /= (g.mx - g.mn);
    thres *= thres;
    int maxpop[kLevels];
    level_maxpop(g, maxpop);
    int invalid_count = 0;
    long long bv = 0, pv = 0;
#pragma omp parallel reduction(+ : invalid_count, bv, pv)
    {
        std::vector<float> dist(k);
        std::vector<std::pair<float, int>> cand;
#pragma omp for schedule(dynamic, 256)
        for (int q = 0; q < n; q++) {
            int* out = lists + (size_t)q * k;
            int reached = 0;
            bool ok = false;
            if (cls[q] < kProposalClasses - 1) ok = box_query(g, q, k, cls[q], thres, maxpop, out, reached, bv, cand);
            if (!ok) {
                int counter;
                bool invalid;
                reached = knn_query(g, q, k, thres, dist.data(), out, counter, invalid, pv);
                if (invalid) invalid_count++;
            }
            certified[q] = ok ? 1 : 0;
            if (level) level[q] = reached;
        }
    }
    *box_visited = bv;
    *plain_visited = pv;
    return invalid_count;
}

// Timed sample of the grid kNN for the CPU baseline: builds the full grid
// (normalisation, cell sort, 8 levels) and answers every `stride`-th query.
// Returns the wall times of both phases (steady_clock, seconds).
void orc_knn_timed(const float* xyz, int n, int k, int stride, double* t_build, double* t_query) {
    auto t0 = std::chrono::steady_clock::now();
    Grid g;
    build_grid(xyz, n, g, kLevels);
    float thres = 1e8f;
    thres /= (g.mx - g.mn);
    thres *= thres;
    auto t1 = std::chrono::steady_clock::now();
    long long sink = 0;
#pragma omp parallel reduction(+ : sink)
    {
        std::vector<float> dist(k);
        std::vector<int> idx(k);
#pragma omp for schedule(dynamic, 64)
        for (int q = 0; q < n; q += stride) {
            int counter;
            bool invalid;
            long long visited = 0;
            knn_query(g, q, k, thres, dist.data(), idx.data(), counter, invalid, visited);
            sink += idx[0];
        }
    }
    auto t2 = std::chrono::steady_clock::now();
    *t_build = std::chrono::duration<double>(t1 - t0).count();
    *t_query = std::chrono::duration<double>(t2 - t1).count() + (sink == 42 ? 1e-300 : 0.0);
}

// Mesh 1-ring lists of GridMeshCuda (GridMeshCuda1.cu:314-511).  Each vertex
// receives the other two corners of every triangle it belongs to, inserted with
// the same admission rule as the grid kNN (strict '<' at slot k, dedup,
// FindPosition).  The reference visits a vertex's triangles in a racy order
// (one atomicExch winner per pass, GridMeshCuda1.cu:110-116); here they are
// visited in ascending triangle order, which fixes the order of equal distances.
// Triangles with any index >= n are skipped (the reference remaps them through
// an out-of-range read, GridMeshCuda1.cu:224-232).
void orc_mesh_1ring(const float* xyz, int n, const uint32_t* tris, int t, int k, int* lists, float* pos,
                    int* perm, float* ext) {
    Grid g;
    build_grid(xyz, n, g, 1);
    std::vector<int> rev(n);
    for (int s = 0; s < n; s++) rev[g.perm[s]] = s;
    // corners grouped by vertex in ascending triangle order
    std::vector<int> cnt(n + 1, 0);
    for (int i = 0; i < t; i++) {
        uint32_t v0 = tris[3 * (size_t)i], v1 = tris[3 * (size_t)i + 1], v2 = tris[3 * (size_t)i + 2];
        if (v0 >= (uint32_t)n || v1 >= (uint32_t)n || v2 >= (uint32_t)n) continue;
        for (int c = 0; c < 3; c++) cnt[rev[tris[3 * (size_t)i + c]] + 1]++;
    }
    for (int v = 0; v < n; v++) cnt[v + 1] += cnt[v];
    std::vector<int> fill(cnt.begin(), cnt.end() - 1), corner((size_t)cnt[n]);
    for (int i = 0; i < t; i++) {
        uint32_t v0 = tris[3 * (size_t)i], v1 = tris[3 * (size_t)i + 1], v2 = tris[3 * (size_t)i + 2];
        if (v0 >= (uint32_t)n || v1 >= (uint32_t)n || v2 >= (uint32_t)n) continue;
        for (int c = 0; c < 3; c++) corner[fill[rev[tris[3 * (size_t)i + c]]]++] = 3 * i + c;
    }
#pragma omp parallel
    {
        std::vector<float> dist(k);
#pragma omp for schedule(dynamic, 1024)
        for (int v = 0; v < n; v++) {
            int* idx = lists + (size_t)v * k;
            for (int i = 0; i < k; i++) { dist[i] = 1e10f; idx[i] = -1; }
            int counter = 0;
            for (int e = cnt[v]; e < cnt[v + 1]; e++) {
                int tri = corner[e] / 3, c1 = corner[e] % 3;
                for (int c2 = 0; c2 < 3; c2++) {
                    if (c2 == c1) continue;
                    int u = rev[tris[3 * (size_t)tri + c2]];
                    float d = dist3(g.x[v], g.y[v], g.z[v], g.x[u], g.y[u], g.z[u]);
                    append(dist.data(), idx, k, counter, d, u);
                }
            }
        }
    }
    for (int s = 0; s < n; s++) {
        pos[s] = g.x[s]; pos[n + s] = g.y[s]; pos[2 * (size_t)n + s] = g.z[s];
        perm[s] = g.perm[s];
    }
    ext[0] = g.mn; ext[1] = g.mx;
}

// EGT filter (calculateEGG_GKNN, EGT_CUDA.cu:172-189): out = lists with the
// rejected entries set to -1.  in and out may alias.
void orc_egt(const float* pos, int n, int k, const int* lists_in, float alpha, int* lists_out) {
    const float* X = pos;
    const float* Y = pos + n;
    const float* Z = pos + 2 * (size_t)n;
#pragma omp parallel
    {
        std::vector<int> row(k);
#pragma omp for schedule(dynamic, 256)
        for (int i = 0; i < n; i++) {
            std::memcpy(row.data(), lists_in + (size_t)i * k, sizeof(int) * k);
            int* out = lists_out + (size_t)i * k;
            for (int j = 0; j < k; j++) out[j] = row[j];
            for (int j = k - 1; j >= 0; j--)
                if (row[j] != -1 && !egt_keep(X, Y, Z, row.data(), j, X[i], Y[i], Z[i], alpha)) out[j] = -1;
        }
    }
}

// Taubin lambda/mu smoothing (taubin_step_GKNN EGT_CUDA.cu:229-276, loop
// EGT_CUDA.cu:559-633) in float, weights exp(-d^2), isRegularized = 0.
void orc_taubin_f32(float* pos, int n, int k, const int* lists, int iters, float lambda, float mu) {
    std::vector<float> tmp(3 * (size_t)n);
    float* in = pos;
    float* out = tmp.data();
    for (int it = 0; it < 2 * iters; it++) {
        const float scale = (it & 1) ? mu : lambda;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            float x1 = in[i], y1 = in[n + i], z1 = in[2 * (size_t)n + i];
            float cx = 0, cy = 0, cz = 0, sum = 0;
            const int* row = lists + (size_t)i * k;
            for (int j = 0; j < k; j++) {
                int m = row[j];
                if (m == -1) continue;
                float x2 = in[m], y2 = in[n + m], z2 = in[2 * (size_t)n + m];
                float w = std::exp(-dist3_taubin(x1, y1, z1, x2, y2, z2));
                cx = acc(cx, w, x2 - x1); cy = acc(cy, w, y2 - y1); cz = acc(cz, w, z2 - z1);
                sum += w;
            }
            if (sum == 0.0f) sum = 1e-8f;
            out[i] = x1 + scale * cx / sum;
            out[n + i] = y1 + scale * cy / sum;
            out[2 * (size_t)n + i] = z1 + scale * cz / sum;
        }
        std::swap(in, out);
    }
    if (in != pos) std::memcpy(pos, in, sizeof(float) * 3 * (size_t)n);
}

// One half-step of taubin_step_GKNN (EGT_CUDA.cu:229-276) over rows [0, rows)
// of a CSR: row i's own position is in[i] and its neighbours are in[col[e]],
// e in [off[i], off[i+1]), list order; positions are float4 (x, y, z, w) as
// the GPU keeps them, m of them (rows <= m).  out: rows float4 (w copied).
// The per-rank step of a row-partitioned smoothing, whose halo positions sit
// in in[rows..m).
void orc_taubin_rows_f32(const float* in, int m, int rows, const int* off, const int* col, float scale,
                         float* out) {
    (void)m;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < rows; i++) {
        const float x1 = in[4 * (size_t)i], y1 = in[4 * (size_t)i + 1], z1 = in[4 * (size_t)i + 2];
        float cx = 0, cy = 0, cz = 0, sum = 0;
        for (int e = off[i]; e < off[i + 1]; e++) {
            const size_t q = 4 * (size_t)col[e];
            const float x2 = in[q], y2 = in[q + 1], z2 = in[q + 2];
            float w = std::exp(-dist3_taubin(x1, y1, z1, x2, y2, z2));
            cx = acc(cx, w, x2 - x1); cy = acc(cy, w, y2 - y1); cz = acc(cz, w, z2 - z1);
            sum += w;
        }
        if (sum == 0.0f) sum = 1e-8f;
        out[4 * (size_t)i] = x1 + scale * cx / sum;
        out[4 * (size_t)i + 1] = y1 + scale * cy / sum;
        out[4 * (size_t)i + 2] = z1 + scale * cz / sum;
        out[4 * (size_t)i + 3] = in[4 * (size_t)i + 3];
    }
}

// Same iteration in double precision (the FP64 oracle).
void orc_taubin_f64(double* pos, int n, int k, const int* lists, int iters, double lambda, double mu) {
    std::vector<double> tmp(3 * (size_t)n);
    double* in = pos;
    double* out = tmp.data();
    for (int it = 0; it < 2 * iters; it++) {
        const double scale = (it & 1) ? mu : lambda;
#pragma omp parallel for schedule(static)
        for (int i = 0; i < n; i++) {
            double x1 = in[i], y1 = in[n + i], z1 = in[2 * (size_t)n + i];
            double cx = 0, cy = 0, cz = 0, sum = 0;
            const int* row = lists + (size_t)i * k;
            for (int j = 0; j < k; j++) {
                int m = row[j];
                if (m == -1) continue;
                double dx = in[m] - x1, dy = in[n + m] - y1, dz = in[2 * (size_t)n + m] - z1;
                double w = std::exp(-(dx * dx + dy * dy + dz * dz));
                cx += w * dx; cy += w * dy; cz += w * dz;
                sum += w;
            }
            if (sum == 0.0) sum = 1e-8;
            out[i] = x1 + scale * cx / sum;
            out[n + i] = y1 + scale * cy / sum;
            out[2 * (size_t)n + i] = z1 + scale * cz / sum;
        }
        std::swap(in, out);
    }
    if (in != pos) std::memcpy(pos, in, sizeof(double) * 3 * (size_t)n);
}

// Unoriented PCA normals (calculateNormal Normal_CUDA.cu:87-144) in sorted
// space: out [3n] SoA.  use_f64 selects the FP64 oracle.
void orc_normals(const float* pos, int n, int k, const int* lists, int use_f64, float* out) {
    const float* X = pos;
    const float* Y = pos + n;
    const float* Z = pos + 2 * (size_t)n;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int i = 0; i < n; i++) {
        if (use_f64) {
            double v[3];
            normal_of<double>(X, Y, Z, lists + (size_t)i * k, k, i, v);
            out[i] = (float)v[0]; out[n + i] = (float)v[1]; out[2 * (size_t)n + i] = (float)v[2];
        } else {
            float v[3];
            normal_of<float>(X, Y, Z, lists + (size_t)i * k, k, i, v);
            out[i] = v[0]; out[n + i] = v[1]; out[2 * (size_t)n + i] = v[2];
        }
    }
}

// Relative gap (l1 - l0) / l2 of the two smallest eigenvalues of each point's
// FP64 covariance (the one normal_of<double> solves): where it is ~0 the normal
// is not defined (any direction in the plane of the two is one).
void orc_normal_gaps(const float* pos, int n, int k, const int* lists, double* gap) {
    const float* X = pos;
    const float* Y = pos + n;
    const float* Z = pos + 2 * (size_t)n;
#pragma omp parallel for schedule(dynamic, 1024)
    for (int i = 0; i < n; i++) {
        const int* row = lists + (size_t)i * k;
        double sx = X[i], sy = Y[i], sz = Z[i];
        int cnt = 1;
        for (int j = 0; j < k; j++) {
            const int m = row[j];
            if (m >= 0) { sx += X[m]; sy += Y[m]; sz += Z[m]; cnt++; }
        }
        const double cx = sx / cnt, cy = sy / cnt, cz = sz / cnt;
        double c00 = 0, c01 = 0, c02 = 0, c11 = 0, c12 = 0, c22 = 0;
        for (int j = 0; j < k; j++) {
            const int m = row[j];
            if (m < 0) continue;
            const double dx = X[m] - cx, dy = Y[m] - cy, dz = Z[m] - cz;
            c00 += dx * dx; c01 += dx * dy; c02 += dx * dz; c11 += dy * dy; c12 += dy * dz; c22 += dz * dz;
        }
        double ev[3], vec[3][3];
        eigen3<double>(c00, c01, c02, c11, c12, c22, ev, vec);
        gap[i] = ev[2] > 0 ? (ev[1] - ev[0]) / ev[2] : 0.0;
    }
}

// Orientation of GetNormals (Normal_CUDA.cu:329-711) on sorted-space normals,
// in place.  Undirected edges (min,max) from the lists with weight
// max(0, 1-|n_u.n_v|) (Normal_CUDA.cu:146-175), deduplicated by the key
// u*n+v and ordered by (weight, key) (Normal_CUDA.cu:363-385).  The spanning
// forest is the minimum one for that total order (Kruskal); the reference's
// Borůvka (CUDA_MST.cu:296-418) computes a minimum forest with its own tie
// rule.  Each tree is traversed breadth-first from the first vertex `u` of its
// lightest edge (for the first tree this is the reference's root,
// Normal_CUDA.cu:438-440), flipping a child whose normal has a negative dot
// product with its parent's (bfs.cu:21-29).  Component sign votes
// (Normal_CUDA.cu:517-711) are applied over list edges that join trees.
// Outputs (optional): parent [n] (-1 roots/untouched), ncomp.
int orc_orient(int n, int k, const int* lists, float* nrm, int* parent) {
    float* NX = nrm;
    float* NY = nrm + n;
    float* NZ = nrm + 2 * (size_t)n;
    struct E { float w; long long key; int u, v; };
    std::vector<E> edges;
    edges.reserve((size_t)n * 8);
    for (int i = 0; i < n; i++)
        for (int j = 0; j < k; j++) {
            int m = lists[(size_t)i * k + j];
            if (m < 0) continue;
            int u = std::min(i, m), v = std::max(i, m);
            float dp = dot3(NX[i], NY[i], NZ[i], NX[m], NY[m], NZ[m]);
            float w = std::fmax(0.0f, 1.0f - std::fabs(dp));
            edges.push_back({w, (long long)u * n + v, u, v});
        }
    std::sort(edges.begin(), edges.end(), [](const E& a, const E& b) { return a.key < b.key; });
    edges.erase(std::unique(edges.begin(), edges.end(), [](const E& a, const E& b) { return a.key == b.key; }),
                edges.end());
    std::stable_sort(edges.begin(), edges.end(), [](const E& a, const E& b) { return a.w < b.w; });
    DSU dsu(n);
    std::vector<std::vector<int>> adj(n);
    for (const E& e : edges) {
        if (e.u == e.v) continue;
        if (dsu.unite(e.u, e.v)) { adj[e.u].push_back(e.v); adj[e.v].push_back(e.u); }
    }
    std::vector<int> comp(n, -1), par(n, -1);
    int ncomp = 0;
    for (const E& e : edges) {
        int root = e.u;
        if (comp[root] >= 0 || adj[root].empty()) continue;
        std::queue<int> qu;
        qu.push(root);
        comp[root] = ncomp;
        while (!qu.empty()) {
            int a = qu.front(); qu.pop();
            for (int b : adj[a]) {
                if (comp[b] >= 0) continue;
                comp[b] = ncomp;
                par[b] = a;
                float dp = dot3(NX[a], NY[a], NZ[a], NX[b], NY[b], NZ[b]);
                if (dp < 0) { NX[b] = -NX[b]; NY[b] = -NY[b]; NZ[b] = -NZ[b]; }
                qu.push(b);
            }
        }
        ncomp++;
    }
    // component votes (componentCounter Normal_CUDA.cu:271-290) and the
    // component-graph BFS (Normal_CUDA.cu:657-711)
    if (ncomp > 1) {
        std::vector<std::vector<int>> votes(ncomp);
        std::vector<std::set<std::pair<int, int>>> cg(ncomp);
        for (int c = 0; c < ncomp; c++) {
            std::vector<int> cnt(ncomp, 0);
            for (int i = 0; i < n; i++) {
                if (comp[i] != c) continue;
                for (int j = 0; j < k; j++) {
                    int m = lists[(size_t)i * k + j];
                    if (m < 0 || comp[m] < 0 || comp[m] == c) continue;
                    float dp = dot3(NX[i], NY[i], NZ[i], NX[m], NY[m], NZ[m]);
                    cnt[comp[m]] += dp > 0 ? 1 : -1;
                }
            }
            for (int o = 0; o < ncomp; o++) {
                if (cnt[o] == 0) continue;
                int orient = cnt[o] > 0 ? 1 : -1;
                cg[c].insert({o, orient});
                cg[o].insert({c, orient});
            }
        }
        std::vector<char> seen(ncomp, 0);
        std::vector<int> flip(ncomp, 0);
        for (int r = 0; r < ncomp; r++) {
            if (seen[r]) continue;
            std::queue<std::pair<int, int>> qq;
            qq.push({r, 1});
            seen[r] = 1;
            while (!qq.empty()) {
                auto [c, o] = qq.front(); qq.pop();
                for (auto [nb, ori] : cg[c]) {
                    if (seen[nb]) continue;
                    if (o * ori < 0) flip[nb] = 1;
                    qq.push({nb, o * ori});
                    seen[nb] = 1;
                }
            }
        }
        for (int i = 0; i < n; i++)
            if (comp[i] >= 0 && flip[comp[i]]) { NX[i] = -NX[i]; NY[i] = -NY[i]; NZ[i] = -NZ[i]; }
    }
    if (parent) std::memcpy(parent, par.data(), sizeof(int) * n);
    return ncomp;
}

// The reference's CPU orienter orient_kruskal (MST.cpp:399-423) with
// Graph::kruskalMST (:297-376), DisjointSets (:185-229) and
// orientSpanningTree (:262-279), in place on host normals.
//   * Edges: for every row i and its first k_use entries m >= 0, the pair
//     (min, max) is kept at its first occurrence (keyed u*n+v; the reference
//     forms that key in 32-bit int arithmetic, which overflows above 46,340
//     points -- this restatement uses 64 bits, the evident intent).  Weight =
//     max(0, 1 - |d|) in double, d the float dot product
//     nx_i*nx_m + ny_i*ny_m + nz_i*nz_m evaluated left to right without
//     fusion.
//   * Kruskal over the edges sorted by (weight, u, v), with a union-find that
//     merges by rank (the second root wins ties and gains a rank) and
//     compresses paths; accepted edges are appended to both endpoints'
//     adjacency lists.
//   * Every union-find root r (parent[r] == r, scanned in index order) starts
//     a depth-first walk with an explicit stack: pop u, then for each
//     unprocessed neighbour v in adjacency order negate n_v when the float
//     dot product of n_u and n_v is negative and push v; u is then processed.
//   key32 != 0 forms the key as the reference does, N * u + v in 32-bit int
//   arithmetic with two's-complement wrap-around (the reference's overflow),
//   so that pairs whose keys collide are dropped as it drops them.
void orient_kruskal_impl(const int* knn, int64_t n, int k, int k_use, float* nx, float* ny, float* nz, int key32) {
    struct Edge { double w; int u, v; };
    auto dotf = [&](int a, int b) {
        const float t = nx[a] * nx[b] + ny[a] * ny[b];
        return t + nz[a] * nz[b];
    };
    std::vector<Edge> edges;
    std::unordered_set<uint64_t> seen;
    seen.reserve((size_t)n * (size_t)std::max(1, k_use));
    for (int64_t i = 0; i < n; i++)
        for (int j = 0; j < k_use; j++) {
            const int m = knn[i * k + j];
            if (m < 0) continue;
            const int u = (int)std::min<int64_t>(i, m), v = (int)std::max<int64_t>(i, m);
            const uint64_t key = key32 ? (uint64_t)(int64_t)(int32_t)((uint32_t)n * (uint32_t)u + (uint32_t)v)
                                       : (uint64_t)u * (uint64_t)n + (uint64_t)v;
            if (!seen.insert(key).second) continue;
            const double d = (double)dotf((int)i, m);
            const double w = std::max(0.0, 1.0 - std::fabs(d));
            edges.push_back({w, u, v});
        }
    std::sort(edges.begin(), edges.end(), [](const Edge& a, const Edge& b) {
        if (a.w != b.w) return a.w < b.w;
        if (a.u != b.u) return a.u < b.u;
        return a.v < b.v;
    });
    std::vector<int> par((size_t)n + 1), rnk((size_t)n + 1, 0);
    std::iota(par.begin(), par.end(), 0);
    auto find = [&](int x) {
        int r = x;
        while (par[r] != r) r = par[r];
        while (par[x] != r) { const int nx_ = par[x]; par[x] = r; x = nx_; }
        return r;
    };
    std::vector<std::vector<int>> adj((size_t)n);
    for (const Edge& e : edges) {
        const int a = find(e.u), b = find(e.v);
        if (a == b) continue;
        adj[e.v].push_back(e.u);
        adj[e.u].push_back(e.v);
        if (rnk[a] > rnk[b]) par[b] = a;
        else par[a] = b;
        if (rnk[a] == rnk[b]) rnk[b]++;
    }
    std::vector<char> processed((size_t)n, 0);
    std::vector<int> stack;
    for (int64_t r = 0; r < n; r++) {
        if (par[r] != r) continue;
        stack.push_back((int)r);
        while (!stack.empty()) {
            const int u = stack.back();
            stack.pop_back();
            for (int v : adj[u]) {
                if (processed[v]) continue;
                if (dotf(u, v) < 0) { nx[v] = -nx[v]; ny[v] = -ny[v]; nz[v] = -nz[v]; }
                stack.push_back(v);
            }
            processed[u] = 1;
        }
    }
}


// getOutputPoints (getOutputPoints.cu:9-63): denormalise and scatter to the
// original order.  pos [3n] sorted SoA -> out [3n] original-order SoA.
void orc_output(const float* pos, const int* perm, const float* ext, int n, float* out) {
    const float d = ext[1] - ext[0];
    for (int s = 0; s < n; s++) {
        int o = perm[s];
        out[o] = denorm(pos[s], d, ext[0]);
        out[n + o] = denorm(pos[n + s], d, ext[0]);
        out[2 * (size_t)n + o] = denorm(pos[2 * (size_t)n + s], d, ext[0]);
    }
}

// Exact brute-force kNN over sorted-space positions, ordered by (distance,
// index), used to check that the grid search is exact.  dist [n*k].
void orc_bruteforce(const float* pos, int n, int k, int* lists, float* dists) {
    const float* X = pos;
    const float* Y = pos + n;
    const float* Z = pos + 2 * (size_t)n;
#pragma omp parallel
    {
        std::vector<std::pair<float, int>> c((size_t)n);
#pragma omp for schedule(dynamic, 64)
        for (int q = 0; q < n; q++) {
            int m = 0;
            for (int p = 0; p < n; p++)
                if (p != q) c[m++] = {dist3(X[q], Y[q], Z[q], X[p], Y[p], Z[p]), p};
            int kk = std::min(k, m);
            std::partial_sort(c.begin(), c.begin() + kk, c.begin() + m);
            for (int j = 0; j < k; j++) {
                lists[(size_t)q * k + j] = j < kk ? c[j].second : -1;
                dists[(size_t)q * k + j] = j < kk ? c[j].first : 1e10f;
            }
        }
    }
}

// Checks the certification rule of the block-selection kNN (product kernel
// k_knn_select) against the reference's ring search (knn_query): for every
// query the cloud's exact k+1 nearest points are found by brute force, and the
// query is "certified" when
//   (1) the k+1 smallest distances are pairwise distinct,
//   (2) the first step s of the ring search (0 = own level-0 cell, s >= 1 =
//       the ring at level s-1) whose face test (decide_more, GridKNNCuda.cu:
//       694-741) stops on the k-th distance exists,
//   (3) the k nearest lie inside the block that step s has visited (level-0
//       cell keys),
//   (4) no cell of the levels visited up to step s holds MAX_PNTS_IN_CUBE
//       points or more (GridKNNCuda.cu:672, 685).
// stats[0] = certified rows, stats[1] = certified rows whose ring-search list
// differs from the k nearest in ascending order (the rule says 0), stats[2] =
// certified rows whose ring-search stop level differs from step s.
void orc_select_check(const float* xyz, int n, int k, long long* stats) {
    Grid g;
    build_grid(xyz, n, g, kLevels);
    float thres = 1e8f;
    thres /= (g.mx - g.mn);
    thres *= thres;
    int maxpop[kLevels];
    for (int L = 0; L < kLevels; L++) {
        maxpop[L] = 0;
        for (size_t c = 0; c + 1 < g.lv[L].start.size(); c++)
            maxpop[L] = std::max(maxpop[L], g.lv[L].start[c + 1] - g.lv[L].start[c]);
    }
    long long certified = 0, wrong = 0, wrong_level = 0;
#pragma omp parallel reduction(+ : certified, wrong, wrong_level)
    {
        std::vector<std::pair<float, int>> c((size_t)n);
        std::vector<float> dist(k);
        std::vector<int> idx(k);
#pragma omp for schedule(dynamic, 64)
        for (int q = 0; q < n; q++) {
            int m = 0;
            for (int p = 0; p < n; p++)
                if (p != q) c[m++] = {dist3(g.x[q], g.y[q], g.z[q], g.x[p], g.y[p], g.z[p]), p};
            if (m < k + 1) continue;
            std::partial_sort(c.begin(), c.begin() + k + 1, c.begin() + m);
            bool ok = true;
            for (int j = 1; j <= k; j++) ok &= c[j - 1].first < c[j].first;
            if (!ok) continue;
            const float T = c[k - 1].first;
            int sf = -1;
            for (int st = 0; st <= kLevels; st++) {
                const int Ls = st == 0 ? 0 : st - 1, o = st == 0 ? 0 : 1;
                if (!decide_more(g, q, Ls, o, k, k, T, thres)) { sf = st; break; }
            }
            if (sf < 0) continue;
            for (int j = 0; j < k && ok; j++) {
                const int p = c[j].second;
                if (sf == 0) {
                    ok = g.cx[p] == g.cx[q] && g.cy[p] == g.cy[q] && g.cz[p] == g.cz[q];
                } else {
                    const int L = sf - 1;
                    ok = std::abs((g.cx[p] >> L) - (g.cx[q] >> L)) <= 1 &&
                         std::abs((g.cy[p] >> L) - (g.cy[q] >> L)) <= 1 &&
                         std::abs((g.cz[p] >> L) - (g.cz[q] >> L)) <= 1;
                }
            }
            for (int L = 0; L <= std::max(sf - 1, 0) && ok; L++) ok = maxpop[L] < kMaxPointsInCube;
            if (!ok) continue;
            certified++;
            int counter;
            bool invalid;
            long long visited = 0;
            const int reached = knn_query(g, q, k, thres, dist.data(), idx.data(), counter, invalid, visited);
            bool same = !invalid;
            for (int j = 0; j < k && same; j++) same = idx[j] == c[j].second;
            if (!same) wrong++;
            if (reached != std::max(sf - 1, 0)) wrong_level++;
        }
    }
    stats[0] = certified;
    stats[1] = wrong;
    stats[2] = wrong_level;
}

// orient_kruskal (MST.cpp:399-423) on host normals, in place; key32 as in
// orient_kruskal_impl.
void orc_orient_kruskal(const int* knn, int64_t n, int k, int k_use, float* nx, float* ny, float* nz, int key32) {
    orient_kruskal_impl(knn, n, k, k_use, nx, ny, nz, key32);
}

}  // extern "C"
