// mhpc oracle: a plain FP64 (OpenMP) CPU restatement of milupHPC's single-rank
// right-hand side.  TEST INFRASTRUCTURE ONLY: it is the checker for the CUDA
// product path.  Only tests/, __graft_entry__.smoke() and bench.py's
// cpu_baseline / reference arm load it; the product library never does.
//
// Every function cites the reference file:line it restates (paths relative to
// the milupHPC project root).  Array layout follows the reference's
// `Particles` SoA: x, y, z, mass are sized num_nodes with tree cells stored
// after the n particles; child[] is 8*num_nodes ints, -1 = empty, and the
// implicit root keeps its eight children in child[0..7]
// (src/subdomain_key_tree/tree.cu:768-1082).
//
// Parity pins: keys, sort order, tree node sets, COM, the v2 walk and the SPH
// pair sums are checked against the reference's own kernels run on the same
// inputs (fixtures under tests/golden/, see tests/golden/make_golden.py).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

extern "C" {

// ---------------------------------------------------------------- bbox ----
// TreeNS::Kernel::computeBoundingBox (tree.cu:302-437) after
// Kernel::resetArrays (device_rhs.cu:24-33): the box is initialised to 0, so
// it always contains the origin, and CUBIC_DOMAINS gives every axis the same
// [min, max].  out = {minX, maxX, minY, maxY, minZ, maxZ}.
void orc_bbox(const double* x, const double* y, const double* z, int n, double* out) {
    double mn = 0.0, mx = 0.0;
    for (int i = 0; i < n; ++i) {
        mn = std::min(mn, std::min(x[i], std::min(y[i], z[i])));
        mx = std::max(mx, std::max(x[i], std::max(y[i], z[i])));
    }
    out[0] = out[2] = out[4] = mn;
    out[1] = out[3] = out[5] = mx;
}

// ---------------------------------------------------------------- keys ----
// Hilbert tables of include/subdomain_key_tree/tree.cuh:66-79 (DirTable) and
// :120-131 (HilbertTable); the tables define the curve, so they are data that
// must be identical.
static const unsigned char kDir[12][8] = {
    {8, 10, 3, 3, 4, 5, 4, 5},  {2, 2, 11, 9, 4, 5, 4, 5},  {7, 6, 7, 6, 8, 10, 1, 1},
    {7, 6, 7, 6, 0, 0, 11, 9},  {0, 8, 1, 11, 6, 8, 6, 11}, {10, 0, 9, 1, 10, 7, 9, 7},
    {10, 4, 9, 4, 10, 2, 9, 3}, {5, 8, 5, 11, 2, 8, 3, 11}, {4, 9, 0, 0, 7, 9, 2, 2},
    {1, 1, 8, 5, 3, 3, 8, 6},   {11, 5, 0, 0, 11, 6, 2, 2}, {1, 1, 4, 10, 3, 3, 7, 10}};
static const unsigned char kHil[12][8] = {
    {0, 7, 3, 4, 1, 6, 2, 5}, {4, 3, 7, 0, 5, 2, 6, 1}, {6, 1, 5, 2, 7, 0, 4, 3},
    {2, 5, 1, 6, 3, 4, 0, 7}, {0, 1, 7, 6, 3, 2, 4, 5}, {6, 7, 1, 0, 5, 4, 2, 3},
    {2, 3, 5, 4, 1, 0, 6, 7}, {4, 5, 3, 2, 7, 6, 0, 1}, {0, 3, 1, 2, 7, 4, 6, 5},
    {2, 1, 3, 0, 5, 6, 4, 7}, {4, 7, 5, 6, 3, 0, 2, 1}, {6, 5, 7, 4, 1, 2, 0, 3}};

// KeyNS::lebesgue2hilbert(key, maxLevel, level) with level == maxLevel
// (tree.cu:40-53).
uint64_t orc_lebesgue2hilbert(uint64_t leb) {
    uint64_t h = 0;
    int dir = 0;
    for (int lvl = 21; lvl > 0; --lvl) {
        int cell = (int)((leb >> (3 * (lvl - 1))) & 7ULL);
        h = (h << 3) + kHil[dir][cell];
        dir = kDir[dir][cell];
    }
    return h;
}

// Tree::getParticleKey (tree.cu:157-240): 21-level top-down bisection of the
// box; octant bit 0/1/2 is set when x/y/z lies BELOW the midpoint
// (tree.cu:182-199) and level l's octant lands at bits 3*(20-l).  The
// reference loop runs a 22nd iteration whose shift count is negative; on the
// GPU that shift yields 0, so the iteration contributes nothing and is
// skipped here.
void orc_keys(const double* x, const double* y, const double* z, int n, const double* bb,
              int curve, uint64_t* keys) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double mnx = bb[0], mxx = bb[1], mny = bb[2], mxy = bb[3], mnz = bb[4], mxz = bb[5];
        uint64_t key = 0;
        for (int level = 0; level < 21; ++level) {
            uint64_t son = 0;
            double mid = 0.5 * (mnx + mxx);
            if (x[i] < mid) { son += 1; mxx = mid; } else { mnx = mid; }
            mid = 0.5 * (mny + mxy);
            if (y[i] < mid) { son += 2; mxy = mid; } else { mny = mid; }
            mid = 0.5 * (mnz + mxz);
            if (z[i] < mid) { son += 4; mxz = mid; } else { mnz = mid; }
            key |= son << (3 * (20 - level));
        }
        keys[i] = curve == 1 ? orc_lebesgue2hilbert(key) : key;
    }
}

// TreeNS::prepareSorting + HelperNS::sortArray (tree.cu:1404-1413,
// helper.cu:150-166): CUB radix SortPairs of (key, index) is stable, so ties
// keep ascending original index.
void orc_sort(const uint64_t* keys, int n, uint64_t* keys_sorted, int* perm) {
    std::vector<int> idx(n);
    for (int i = 0; i < n; ++i) idx[i] = i;
    std::stable_sort(idx.begin(), idx.end(), [&](int a, int b) { return keys[a] < keys[b]; });
    for (int i = 0; i < n; ++i) { perm[i] = idx[i]; keys_sorted[i] = keys[idx[i]]; }
}

// ---------------------------------------------------------------- tree ----
// TreeNS::Kernel::buildTree (tree.cu:768-1082) restated as sequential
// insertion in particle order: descend by FP64 midpoint compares, split a
// leaf into new cells (numbered from n upward) until the two particles
// separate.  A new cell's x,y,z is the geometric centre of its box
// (tree.cu:995-1001), its level is its depth (root children = 1), a
// particle's level is its parent's level + 1.  child must hold 8*num_nodes
// ints and level num_nodes ints.  Returns the number of nodes used
// (n + cells), -1 if the node pool is exhausted, -2 if two particles could not
// be separated within 64 levels.
int orc_tree_build(const double* px, const double* py, const double* pz, int n, int num_nodes,
                   const double* bb, int* child, int* level, double* x, double* y, double* z,
                   double* mass) {
    for (long i = 0; i < 8L * num_nodes; ++i) child[i] = -1;
    for (int i = 0; i < num_nodes; ++i) level[i] = -1;
    for (int i = n; i < num_nodes; ++i) { x[i] = y[i] = z[i] = mass[i] = 0.0; }
    int next = n;
    for (int p = 0; p < n; ++p) {
        double mnx = bb[0], mxx = bb[1], mny = bb[2], mxy = bb[3], mnz = bb[4], mxz = bb[5];
        auto step = [&](double qx, double qy, double qz, bool shrink) {
            int son = 0;
            double mid = 0.5 * (mnx + mxx);
            if (qx < mid) { son += 1; if (shrink) mxx = mid; } else if (shrink) mnx = mid;
            mid = 0.5 * (mny + mxy);
            if (qy < mid) { son += 2; if (shrink) mxy = mid; } else if (shrink) mny = mid;
            mid = 0.5 * (mnz + mxz);
            if (qz < mid) { son += 4; if (shrink) mxz = mid; } else if (shrink) mnz = mid;
            return son;
        };
        int temp = 0, lvl = 0;
        int son = step(px[p], py[p], pz[p], true);
        int ch = child[8 * temp + son];
        while (ch >= n) {
            temp = ch; ++lvl;
            son = step(px[p], py[p], pz[p], true);
            ch = child[8 * temp + son];
        }
        if (ch == -1) {
            child[8 * temp + son] = p;
            level[p] = lvl + 1;
            continue;
        }
        int q = ch;
        for (;;) {
            if (next >= num_nodes) return -1;
            int cell = next++;
            child[8 * temp + son] = cell;
            ++lvl;
            if (lvl > 64) return -2;
            x[cell] = 0.5 * (mnx + mxx);
            y[cell] = 0.5 * (mny + mxy);
            z[cell] = 0.5 * (mnz + mxz);
            level[cell] = lvl;
            level[q] += 1;
            int sq = step(px[q], py[q], pz[q], false);
            child[8 * cell + sq] = q;
            temp = cell;
            son = step(px[p], py[p], pz[p], true);
            if (child[8 * cell + son] == -1) break;
        }
        child[8 * temp + son] = p;
        level[p] = lvl + 1;
    }
    return next;
}

// TreeNS::Kernel::calculateCentersOfMass (tree.cu:1416-1497) as launched by
// Miluphpc::parallel_pseudoParticles (miluphpc.cpp:1205-1210): for level
// max_level..1, each cell of that level sums its children in octant order.
// The reference loops levels 21..1 only; max_level lets a caller include the
// deeper cells that near-coincident particles create.
void orc_com(const int* child, const int* level, int n, int nodes, int max_level, double* x,
             double* y, double* z, double* mass) {
    for (int L = max_level; L > 0; --L) {
#pragma omp parallel for schedule(static)
        for (int i = n; i < nodes; ++i) {
            if (level[i] != L) continue;
            double m = 0, sx = 0, sy = 0, sz = 0;
            for (int c = 0; c < 8; ++c) {
                int ch = child[8 * i + c];
                if (ch != -1) {
                    sx += x[ch] * mass[ch];
                    sy += y[ch] * mass[ch];
                    sz += z[ch] * mass[ch];
                    m += mass[ch];
                }
            }
            if (m > 0.) { sx /= m; sy /= m; sz /= m; }
            mass[i] = m; x[i] = sx; y[i] = sy; z[i] = sz;
        }
    }
}

// Canonical node set: for every cell reachable from the root, its Lebesgue
// key prefix (level digits, leading octant first, in the same bit convention
// as the keys) and level.  Used to compare trees whose node numbering differs
// ("equal as sets of (key, level)").  Writes up to cap pairs, returns count.
int orc_tree_nodeset(const int* child, int n, uint64_t* prefixes, int* levels, int cap) {
    struct Item { int node; uint64_t prefix; int level; };
    std::vector<Item> stack;
    int cnt = 0;
    for (int c = 0; c < 8; ++c) {
        int ch = child[c];
        if (ch >= n) stack.push_back({ch, (uint64_t)c, 1});
    }
    while (!stack.empty()) {
        Item it = stack.back();
        stack.pop_back();
        if (cnt < cap) { prefixes[cnt] = it.prefix; levels[cnt] = it.level; }
        ++cnt;
        for (int c = 0; c < 8; ++c) {
            int ch = child[8 * it.node + c];
            if (ch >= n) stack.push_back({ch, (it.prefix << 3) | (uint64_t)c, it.level + 1});
        }
    }
    return cnt;
}

// ------------------------------------------------------------- gravity ----
// Gravity::Kernel::computeForces_v2 (gravity.cu:726-903), the default
// gravityForceVersion 0.  Warps take 32 consecutive entries of the sorted
// order and share one stack: a child is accepted if it is a leaf (index < n)
// or if EVERY lane has dp <= r, r = |d|^2 + eps2, dp = 0.25*depth with
// depth(root children) = radius^2/theta.  Root children are always opened;
// a root child that is a leaf is pushed like a cell and contributes through
// its own child slots (empty for every particle but particle 0).
// Accumulation order follows the reference's LIFO stack.  With stride > 1 only
// every stride-th warp group is computed (a bounded sample for timing).
void orc_gravity_v2_sample(const double* x, const double* y, const double* z, const double* mass,
                           const int* child, const int* sorted, int n, double radius, double theta,
                           double eps2, double* gax, double* gay, double* gaz, int stride) {
    const int ngroups = (n + 31) / 32;
    if (stride < 1) stride = 1;
#pragma omp parallel for schedule(dynamic, 4)
    for (int g = 0; g < ngroups; g += stride) {
        const int base = g * 32;
        const int lanes = std::min(32, n - base);
        double px[32], py[32], pz[32], ax[32], ay[32], az[32], r[32];
        for (int l = 0; l < lanes; ++l) {
            int s = sorted[base + l];
            px[l] = x[s]; py[l] = y[s]; pz[l] = z[s];
            ax[l] = ay[l] = az[l] = 0.0;
        }
        std::vector<int> snode(4096);
        std::vector<double> sdepth(4096);
        int top = -1;
        for (int i = 0; i < 8; ++i)
            if (child[i] != -1) { ++top; snode[top] = child[i]; sdepth[top] = radius * radius / theta; }
        while (top >= 0) {
            int node = snode[top];
            double dp = 0.25 * sdepth[top];
            for (int i = 0; i < 8; ++i) {
                int ch = child[8 * node + i];
                if (ch < 0) continue;
                bool all = true;
                for (int l = 0; l < lanes; ++l) {
                    double dx = x[ch] - px[l], dy = y[ch] - py[l], dz = z[ch] - pz[l];
                    double rr = dx * dx + eps2;
                    rr += dy * dy;
                    rr += dz * dz;
                    r[l] = rr;
                    if (!(dp <= rr)) all = false;
                }
                if (ch < n || all) {
                    for (int l = 0; l < lanes; ++l) {
                        double rr = r[l];
                        if (rr > 0.) rr = 1.0 / std::sqrt(rr);
                        double f = mass[ch] * rr * rr * rr;
                        ax[l] += f * (x[ch] - px[l]);
                        ay[l] += f * (y[ch] - py[l]);
                        az[l] += f * (z[ch] - pz[l]);
                    }
                } else {
                    if (top + 1 >= (int)snode.size()) { snode.resize(2 * snode.size()); sdepth.resize(2 * sdepth.size()); }
                    snode[top] = ch;
                    sdepth[top] = dp;
                    ++top;
                }
            }
            --top;
        }
        for (int l = 0; l < lanes; ++l) {
            int s = sorted[base + l];
            gax[s] = ax[l]; gay[s] = ay[l]; gaz[s] = az[l];
        }
    }
}

void orc_gravity_v2(const double* x, const double* y, const double* z, const double* mass,
                    const int* child, const int* sorted, int n, double radius, double theta,
                    double eps2, double* gax, double* gay, double* gaz) {
    orc_gravity_v2_sample(x, y, z, mass, child, sorted, n, radius, theta, eps2, gax, gay, gaz, 1);
}

// Gravity::Kernel::computeForces_v1 (gravity.cu:252-396), gravityForceVersion
// 2: per-particle stack walk, accept a child if it is a leaf or
// d^2 * theta^2 > cellSize(depth), cellSize(1) = radius^2 and quartering per
// level; the particle itself is skipped.  Also returns, per particle, the
// number of accepted interactions (used as the walk's work unit).
void orc_gravity_v1(const double* x, const double* y, const double* z, const double* mass,
                    const int* child, int n, double radius, double theta, double eps2,
                    double* gax, double* gay, double* gaz, int* ninter) {
    const double th2 = theta * theta;
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        double ax = 0, ay = 0, az = 0;
        int cnt = 0;
        struct Fr { int node; int c; double cs; };
        Fr st[256];
        int sp = 0;
        st[0] = {-1, 0, radius * radius};
        // node -1 stands for the implicit root whose children are child[0..7]
        while (sp >= 0) {
            Fr& f = st[sp];
            if (f.c >= 8) { --sp; continue; }
            int ch = f.node < 0 ? child[f.c] : child[8 * f.node + f.c];
            f.c++;
            if (ch == -1 || ch == i) continue;
            double dx = x[ch] - x[i], dy = y[ch] - y[i], dz = z[ch] - z[i];
            double d = dx * dx + eps2;
            d += dy * dy;
            d += dz * dz;
            if (ch < n || d * th2 > f.cs) {
                double s = std::sqrt(d);
                double ff = mass[ch] / (s * s * s);
                ax += ff * dx; ay += ff * dy; az += ff * dz;
                ++cnt;
            } else if (sp + 1 < 256) {
                double cs = f.cs * 0.25;
                st[++sp] = {ch, 0, cs};
            }
        }
        gax[i] = ax; gay[i] = ay; gaz[i] = az;
        if (ninter) ninter[i] = cnt;
    }
}

// FP64 direct summation with the same Plummer softening (truth reference):
// a_i = sum_j m_j d_ij / (|d_ij|^2 + eps2)^{3/2}, for the listed targets.
void orc_direct(const double* x, const double* y, const double* z, const double* mass, int n,
                const int* targets, int nt, double eps2, double* gax, double* gay, double* gaz,
                double* pot) {
#pragma omp parallel for schedule(dynamic, 4)
    for (int t = 0; t < nt; ++t) {
        int i = targets[t];
        double ax = 0, ay = 0, az = 0, ph = 0;
        for (int j = 0; j < n; ++j) {
            if (j == i) continue;
            double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
            double r2 = dx * dx + dy * dy + dz * dz + eps2;
            double ri = 1.0 / std::sqrt(r2);
            double f = mass[j] * ri * ri * ri;
            ax += f * dx; ay += f * dy; az += f * dz;
            ph -= mass[j] * ri;
        }
        gax[t] = ax; gay[t] = ay; gaz[t] = az;
        if (pot) pot[t] = ph;
    }
}


// ------------------------------------------------- mixed-path oracle -----
// Traceless quadrupole moments of every cell about its centre of mass,
// Q_ab = sum_k m_k (3 s_a s_b - |s|^2 delta_ab), s = x_k - com, gathered from
// the children by the parallel-axis rule (leaves carry no moment).  Layout
// q[6*node + {xx, xy, xz, yy, yz, zz}].  This is not in the reference: it is
// the FP64 statement of the mixed path's multipole pass.
void orc_quad(const int* child, const int* level, int n, int nodes, int max_level,
              const double* x, const double* y, const double* z, const double* mass, double* q) {
    for (int i = 0; i < 6 * nodes; ++i) q[i] = 0.0;
    for (int L = max_level; L > 0; --L) {
#pragma omp parallel for schedule(static)
        for (int i = n; i < nodes; ++i) {
            if (level[i] != L) continue;
            double t[6] = {0, 0, 0, 0, 0, 0};
            for (int c = 0; c < 8; ++c) {
                int ch = child[8 * i + c];
                if (ch == -1) continue;
                double s[3] = {x[ch] - x[i], y[ch] - y[i], z[ch] - z[i]};
                double s2 = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
                double m = mass[ch];
                t[0] += m * (3 * s[0] * s[0] - s2); t[1] += m * 3 * s[0] * s[1];
                t[2] += m * 3 * s[0] * s[2];        t[3] += m * (3 * s[1] * s[1] - s2);
                t[4] += m * 3 * s[1] * s[2];        t[5] += m * (3 * s[2] * s[2] - s2);
                if (ch >= n) for (int k = 0; k < 6; ++k) t[k] += q[6 * ch + k];
            }
            for (int k = 0; k < 6; ++k) q[6 * i + k] = t[k];
        }
    }
}

// Group walk of the mixed path in FP64: groups of `gsize` consecutive sorted
// particles; a cell at level L is accepted for the group when, for every
// particle p of the group,
//   edge_L^2 / theta <= |com - p|^2
// (edge_L = 2 radius / 2^L; the softening takes no part in the decision): the
// reference's squared-ratio criterion with
// computeForces_v2's all-lanes vote, applied to every level (root children
// included); accepted cells add their monopole and, if q is given,
// quadrupole term.  Leaves are exact.  ninter (per particle) receives the
// number of accepted nodes.
// With crit != null a cell is accepted when crit[cell] <= min |com - p|^2
// (per-cell thresholds, e.g. from orc_cell_bmax2).
void orc_gravity_group_crit(const double* x, const double* y, const double* z, const double* mass,
                            const double* q, const int* child, const int* level, const int* sorted,
                            int n, int gsize, double radius, double theta, double eps2, double* gax,
                            double* gay, double* gaz, int* ninter, const double* crit);

void orc_gravity_group(const double* x, const double* y, const double* z, const double* mass,
                       const double* q, const int* child, const int* level, const int* sorted,
                       int n, int gsize, double radius, double theta, double eps2, double* gax,
                       double* gay, double* gaz, int* ninter) {
    orc_gravity_group_crit(x, y, z, mass, q, child, level, sorted, n, gsize, radius, theta, eps2, gax, gay,
                           gaz, ninter, nullptr);
}

// Squared distance from every cell's centre of mass to the farthest corner of
// the bounding box of its particles (children first, leaves are points).
void orc_cell_bmax2(const int* child, const int* level, int n, int nodes, int max_level,
                    const double* x, const double* y, const double* z, double* bmax2) {
    std::vector<double> lo(3 * (size_t)nodes), hi(3 * (size_t)nodes);
    for (int i = 0; i < n; ++i) {
        lo[3 * i] = hi[3 * i] = x[i]; lo[3 * i + 1] = hi[3 * i + 1] = y[i]; lo[3 * i + 2] = hi[3 * i + 2] = z[i];
    }
    for (int L = max_level; L > 0; --L) {
        for (int i = n; i < nodes; ++i) {
            if (level[i] != L) continue;
            double l3[3] = {1e300, 1e300, 1e300}, h3[3] = {-1e300, -1e300, -1e300};
            for (int c = 0; c < 8; ++c) {
                int ch = child[8 * i + c];
                if (ch < 0) continue;
                for (int d = 0; d < 3; ++d) {
                    l3[d] = std::min(l3[d], lo[3 * (size_t)ch + d]);
                    h3[d] = std::max(h3[d], hi[3 * (size_t)ch + d]);
                }
            }
            double c3[3] = {x[i], y[i], z[i]}, b = 0;
            for (int d = 0; d < 3; ++d) {
                lo[3 * (size_t)i + d] = l3[d]; hi[3 * (size_t)i + d] = h3[d];
                double e = std::max(c3[d] - l3[d], h3[d] - c3[d]);
                b += e * e;
            }
            bmax2[i] = b;
        }
    }
}

void orc_gravity_group_crit(const double* x, const double* y, const double* z, const double* mass,
                            const double* q, const int* child, const int* level, const int* sorted,
                            int n, int gsize, double radius, double theta, double eps2, double* gax,
                            double* gay, double* gaz, int* ninter, const double* crit) {
    const int ngroups = (n + gsize - 1) / gsize;
#pragma omp parallel for schedule(dynamic, 4)
    for (int g = 0; g < ngroups; ++g) {
        const int base = g * gsize;
        const int lanes = std::min(gsize, n - base);
        std::vector<int> stack;
        for (int i = 0; i < 8; ++i) if (child[i] != -1) stack.push_back(child[i]);
        std::vector<int> acc_nodes;
        while (!stack.empty()) {
            int nd = stack.back(); stack.pop_back();
            if (nd < n) { acc_nodes.push_back(nd); continue; }
            double d2 = 1e300;
            for (int l = 0; l < lanes; ++l) {
                int s = sorted[base + l];
                double dx = x[nd] - x[s], dy = y[nd] - y[s], dz = z[nd] - z[s];
                d2 = std::min(d2, dx * dx + dy * dy + dz * dz);
            }
            double edge = 2.0 * radius * std::ldexp(1.0, -level[nd]);
            double cr = crit ? crit[nd] : edge * edge / theta;
            if (cr <= d2) { acc_nodes.push_back(nd); continue; }
            for (int i = 0; i < 8; ++i) if (child[8 * nd + i] != -1) stack.push_back(child[8 * nd + i]);
        }
        for (int l = 0; l < lanes; ++l) {
            int s = sorted[base + l];
            double ax = 0, ay = 0, az = 0;
            for (int nd : acc_nodes) {
                double R[3] = {x[s] - x[nd], y[s] - y[nd], z[s] - z[nd]};
                double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2] + eps2;
                if (nd == s) continue;
                double ri = 1.0 / std::sqrt(r2), ri2 = ri * ri, ri3 = ri * ri2;
                double m = mass[nd];
                ax -= m * ri3 * R[0]; ay -= m * ri3 * R[1]; az -= m * ri3 * R[2];
                if (q && nd >= n) {
                    const double* Q = q + 6 * nd;
                    double QR[3] = {Q[0] * R[0] + Q[1] * R[1] + Q[2] * R[2],
                                    Q[1] * R[0] + Q[3] * R[1] + Q[4] * R[2],
                                    Q[2] * R[0] + Q[4] * R[1] + Q[5] * R[2]};
                    double RQR = R[0] * QR[0] + R[1] * QR[1] + R[2] * QR[2];
                    double ri5 = ri3 * ri2, ri7 = ri5 * ri2;
                    ax += QR[0] * ri5 - 2.5 * RQR * R[0] * ri7;
                    ay += QR[1] * ri5 - 2.5 * RQR * R[1] * ri7;
                    az += QR[2] * ri5 - 2.5 * RQR * R[2] * ri7;
                }
            }
            gax[s] = ax; gay[s] = ay; gaz[s] = az;
            if (ninter) ninter[s] = (int)acc_nodes.size();
        }
    }
}

// Interaction-list walk of the mixed path in FP64: groups of `gsize`
// consecutive sorted particles, each split into `nsub` sub-boxes of gsize/nsub
// consecutive particles (axis-aligned bounding boxes of their positions).  A
// cell is accepted for the group when, for every sub-box b,
//   edge_L^2 / theta <= dist(com, box_b)^2
// (edge_L = 2 radius / 2^L, distance 0 inside the box); otherwise it is
// opened.  Leaves are always accepted (exact).  Accepted cells add their
// monopole and quadrupole terms, accepted leaves their monopole; the softened
// distance |R|^2 + eps2 is used for the interaction, and eps2_i = eps2 +
// (h_factor h_i)^2 per particle when h is given.  ninter receives the number
// of accepted nodes, nquad the number of accepted cells (per particle).
// With amag != null the relative criterion is added (Springel 2005, the
// GADGET-2 opening rule, for a group): a cell of mass M and edge l is
// accepted only if, for every sub-box b with smallest previous |a| a_b,
//   M l^lpow <= alpha a_b dist(com, box_b)^(lpow + 2),
// i.e. the first neglected multipole term stays below alpha times the
// particle's own acceleration; the geometric condition with theta stays as a
// safety bound.  a_b is floored at kRelFloor times the largest previous |a| of
// the sub-box: near a potential minimum |a| tends to zero and the unfloored
// rule would open the whole tree for that group (the device kernel applies
// the same floor).  amag is indexed like x (original order).
static const double kRelFloor = 0.1;

static void gravity_boxes_impl(const double* x, const double* y, const double* z, const double* mass,
                               const double* q, const int* child, const int* level, const int* sorted,
                               int n, int gsize, int nsub, double radius, double theta, double eps2,
                               const double* h, double h_factor, const double* amag, double alpha, int lpow,
                               double* gax, double* gay, double* gaz, int* ninter, int* nquad,
                               double mono_alpha = 0.0) {
    const int ngroups = (n + gsize - 1) / gsize;
    const int w = gsize / nsub;
#pragma omp parallel for schedule(dynamic, 4)
    for (int g = 0; g < ngroups; ++g) {
        const int base = g * gsize;
        const int lanes = std::min(gsize, n - base);
        // sub-box b covers group members [b*w, (b+1)*w); members past n
        // repeat the last particle (as the device kernel loads them)
        std::vector<double> lo(3 * nsub, 1e300), hi(3 * nsub, -1e300), amin(nsub, 1e300), amax(nsub, 0.0);
        for (int j = 0; j < gsize; ++j) {
            const int s = sorted[std::min(base + j, n - 1)];
            const int b = j / w;
            if (amag) { amin[b] = std::min(amin[b], amag[s]); amax[b] = std::max(amax[b], amag[s]); }
            const double p[3] = {x[s], y[s], z[s]};
            for (int d = 0; d < 3; ++d) {
                lo[3 * b + d] = std::min(lo[3 * b + d], p[d]);
                hi[3 * b + d] = std::max(hi[3 * b + d], p[d]);
            }
        }
        if (amag)
            for (int b = 0; b < nsub; ++b) amin[b] = std::max(amin[b], kRelFloor * amax[b]);
        std::vector<int> stack;
        for (int i = 0; i < 8; ++i) if (child[i] != -1) stack.push_back(child[i]);
        std::vector<int> acc_nodes;
        std::vector<char> use_quad;
        int ncell = 0, nquad_g = 0;
        while (!stack.empty()) {
            int nd = stack.back(); stack.pop_back();
            if (nd < n) { acc_nodes.push_back(nd); use_quad.push_back(0); continue; }
            const double edge = 2.0 * radius * std::ldexp(1.0, -level[nd]);
            const double cr = edge * edge / theta;
            const double c[3] = {x[nd], y[nd], z[nd]};
            bool ok = true;
            for (int b = 0; b < nsub && ok; ++b) {
                double d2 = 0.0;
                for (int d = 0; d < 3; ++d) {
                    const double e = std::max(std::max(lo[3 * b + d] - c[d], c[d] - hi[3 * b + d]), 0.0);
                    d2 += e * e;
                }
                ok = cr <= d2;
                if (ok && amag) {
                    const double lp = lpow == 3 ? edge * edge * edge : edge * edge;
                    const double dp = lpow == 3 ? d2 * d2 * std::sqrt(d2) : d2 * d2;
                    ok = mass[nd] * lp <= alpha * amin[b] * dp;
                }
            }
            if (ok) {
                // monopole only when the quadrupole term M l^2 / d^4 stays below
                // mono_alpha |a| for every sub-box (mono_alpha = 0: always quadrupole)
                bool quad = true;
                if (mono_alpha > 0.0 && amag) {
                    quad = false;
                    for (int b = 0; b < nsub && !quad; ++b) {
                        double d2 = 0.0;
                        for (int d = 0; d < 3; ++d) {
                            const double e = std::max(std::max(lo[3 * b + d] - c[d], c[d] - hi[3 * b + d]), 0.0);
                            d2 += e * e;
                        }
                        quad = !(mass[nd] * edge * edge <= mono_alpha * amin[b] * d2 * d2);
                    }
                }
                acc_nodes.push_back(nd); use_quad.push_back(quad ? 1 : 0); ++ncell; nquad_g += quad;
                continue;
            }
            for (int i = 0; i < 8; ++i) if (child[8 * nd + i] != -1) stack.push_back(child[8 * nd + i]);
        }
        for (int l = 0; l < lanes; ++l) {
            const int s = sorted[base + l];
            double e2 = eps2;
            if (h && h_factor > 0.0) { const double e = h_factor * h[s]; e2 += e * e; }
            double ax = 0, ay = 0, az = 0;
            for (size_t t = 0; t < acc_nodes.size(); ++t) {
                const int nd = acc_nodes[t];
                if (nd == s) continue;
                double R[3] = {x[s] - x[nd], y[s] - y[nd], z[s] - z[nd]};
                double r2 = R[0] * R[0] + R[1] * R[1] + R[2] * R[2] + e2;
                double ri = 1.0 / std::sqrt(r2), ri2 = ri * ri, ri3 = ri * ri2;
                double m = mass[nd];
                ax -= m * ri3 * R[0]; ay -= m * ri3 * R[1]; az -= m * ri3 * R[2];
                if (q && nd >= n && use_quad[t]) {
                    const double* Q = q + 6 * nd;
                    double QR[3] = {Q[0] * R[0] + Q[1] * R[1] + Q[2] * R[2],
                                    Q[1] * R[0] + Q[3] * R[1] + Q[4] * R[2],
                                    Q[2] * R[0] + Q[4] * R[1] + Q[5] * R[2]};
                    double RQR = R[0] * QR[0] + R[1] * QR[1] + R[2] * QR[2];
                    double ri5 = ri3 * ri2, ri7 = ri5 * ri2;
                    ax += QR[0] * ri5 - 2.5 * RQR * R[0] * ri7;
                    ay += QR[1] * ri5 - 2.5 * RQR * R[1] * ri7;
                    az += QR[2] * ri5 - 2.5 * RQR * R[2] * ri7;
                }
            }
            gax[s] = ax; gay[s] = ay; gaz[s] = az;
            if (ninter) ninter[s] = (int)acc_nodes.size();
            if (nquad) nquad[s] = mono_alpha > 0.0 ? nquad_g : ncell;
        }
    }
}

void orc_gravity_boxes(const double* x, const double* y, const double* z, const double* mass,
                       const double* q, const int* child, const int* level, const int* sorted,
                       int n, int gsize, int nsub, double radius, double theta, double eps2,
                       const double* h, double h_factor, double* gax, double* gay, double* gaz,
                       int* ninter, int* nquad) {
    gravity_boxes_impl(x, y, z, mass, q, child, level, sorted, n, gsize, nsub, radius, theta, eps2, h, h_factor,
                       nullptr, 0.0, 2, gax, gay, gaz, ninter, nquad);
}

void orc_gravity_boxes_rel(const double* x, const double* y, const double* z, const double* mass,
                           const double* q, const int* child, const int* level, const int* sorted,
                           int n, int gsize, int nsub, double radius, double theta, double eps2,
                           const double* h, double h_factor, const double* amag, double alpha, int lpow,
                           double* gax, double* gay, double* gaz, int* ninter, int* nquad) {
    gravity_boxes_impl(x, y, z, mass, q, child, level, sorted, n, gsize, nsub, radius, theta, eps2, h, h_factor,
                       amag, alpha, lpow, gax, gay, gaz, ninter, nquad);
}

// ----------------------------------------------------------------- SPH ----
// Neighbour sets of SPH::fixedRadiusNN (sph.cu:93-281): j != i with
// d^2 < h_i^2 and d^2 < h_j^2.  The tree walk there is conservative, so the
// set equals this brute-force one (uniform cell grid of edge max h).  Output
// is CSR with neighbours ascending: off[n+1], nbr[off[n]].  When nbr is null
// only off[] (counts) is produced.
void orc_frnn(const double* x, const double* y, const double* z, const double* h, int n,
              long* off, int* nbr) {
    double hmax = 0, mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
    for (int i = 0; i < n; ++i) {
        hmax = std::max(hmax, h[i]);
        mn[0] = std::min(mn[0], x[i]); mx[0] = std::max(mx[0], x[i]);
        mn[1] = std::min(mn[1], y[i]); mx[1] = std::max(mx[1], y[i]);
        mn[2] = std::min(mn[2], z[i]); mx[2] = std::max(mx[2], z[i]);
    }
    double cell = hmax > 0 ? hmax : 1.0;
    int dims[3];
    for (int d = 0; d < 3; ++d) {
        double span = mx[d] - mn[d];
        long k = (long)(span / cell) + 1;
        if (k > 1024) { k = 1024; }
        dims[d] = (int)k;
    }
    double csz[3];
    for (int d = 0; d < 3; ++d) csz[d] = std::max((mx[d] - mn[d]) / dims[d], cell);
    for (int d = 0; d < 3; ++d) dims[d] = std::max(1, (int)((mx[d] - mn[d]) / csz[d]) + 1);
    long ncell = (long)dims[0] * dims[1] * dims[2];
    std::vector<int> cid(n), cstart(ncell + 1, 0), order(n);
    for (int i = 0; i < n; ++i) {
        int c0 = std::min(dims[0] - 1, (int)((x[i] - mn[0]) / csz[0]));
        int c1 = std::min(dims[1] - 1, (int)((y[i] - mn[1]) / csz[1]));
        int c2 = std::min(dims[2] - 1, (int)((z[i] - mn[2]) / csz[2]));
        cid[i] = (c2 * dims[1] + c1) * dims[0] + c0;
        cstart[cid[i] + 1]++;
    }
    for (long c = 0; c < ncell; ++c) cstart[c + 1] += cstart[c];
    {
        std::vector<int> fill(cstart.begin(), cstart.end() - 1);
        for (int i = 0; i < n; ++i) order[fill[cid[i]]++] = i;
    }
    std::vector<int> cnt(n);
    auto visit = [&](int i, bool write, long o) {
        int c0 = cid[i] % dims[0], c1 = (cid[i] / dims[0]) % dims[1], c2 = cid[i] / (dims[0] * dims[1]);
        int k = 0;
        std::vector<int> tmp;
        for (int a = std::max(0, c2 - 1); a <= std::min(dims[2] - 1, c2 + 1); ++a)
            for (int b = std::max(0, c1 - 1); b <= std::min(dims[1] - 1, c1 + 1); ++b)
                for (int c = std::max(0, c0 - 1); c <= std::min(dims[0] - 1, c0 + 1); ++c) {
                    long cc = ((long)a * dims[1] + b) * dims[0] + c;
                    for (int q = cstart[cc]; q < cstart[cc + 1]; ++q) {
                        int j = order[q];
                        if (j == i) continue;
                        double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
                        double d = dx * dx + dy * dy + dz * dz;
                        if (d < h[i] * h[i] && d < h[j] * h[j]) {
                            if (write) tmp.push_back(j);
                            ++k;
                        }
                    }
                }
        if (write) {
            std::sort(tmp.begin(), tmp.end());
            for (size_t t = 0; t < tmp.size(); ++t) nbr[o + t] = tmp[t];
        }
        return k;
    };
#pragma omp parallel for schedule(dynamic, 256)
    for (int i = 0; i < n; ++i) cnt[i] = visit(i, false, 0);
    off[0] = 0;
    for (int i = 0; i < n; ++i) off[i + 1] = off[i] + cnt[i];
    if (nbr) {
#pragma omp parallel for schedule(dynamic, 256)
        for (int i = 0; i < n; ++i) visit(i, true, off[i]);
    }
}

// SmoothingKernel::{spiky, cubicSpline, wendlandc2, wendlandc4, wendlandc6},
// 3-D forms (kernel.cu:14-183), support radius = sml; type 0 spiky, 1 cubic
// spline (f = 8/(pi h^3), split at q = 1/2), 2/3/4 Wendland C2/C4/C6 (Dehnen &
// Aly 2012; the C4 derivative as the reference writes it).  dWdx = dWdr/r * dx
// (NaN at r = 0, as in the reference; only the self-density call hits r = 0
// and it ignores dWdx).
static inline void skern(int type, double* W, double dWdx[3], double* dWdr, const double dx[3], double sml) {
    double r = std::sqrt(dx[0] * dx[0] + dx[1] * dx[1] + dx[2] * dx[2]);
    double q = r / sml;
    *W = 0;
    *dWdr = 0;
    switch (type) {
        case 0:
            if (q > 1) { *W = 0; }
            else if (q >= 0.0) {
                *W = 15. / (M_PI * sml * sml * sml) * (1 - q) * (1 - q) * (1 - q);
                *dWdr = -45 / (M_PI * sml * sml * sml * sml) * (1 - q) * (1 - q);
            }
            break;
        case 1: {
            double f = 8. / M_PI * 1. / (sml * sml * sml);
            if (q > 1) { *W = 0; *dWdr = 0.0; }
            else if (q > 0.5) { *W = 2. * f * (1. - q) * (1. - q) * (1 - q); *dWdr = -6. * f * 1. / sml * (1. - q) * (1. - q); }
            else { *W = f * (6. * q * q * q - 6. * q * q + 1.); *dWdr = 6. * f / sml * (3 * q * q - 2 * q); }
        } break;
        case 2:
            if (r <= sml) {
                *W = 21. / (2 * M_PI * sml * sml * sml) * (1 - q) * (1 - q) * (1 - q) * (1 - q) * (1 + 4 * q) * (q < 1);
                *dWdr = -210. / (M_PI * sml * sml * sml * sml) * q * (1 - q) * (1 - q) * (1 - q) * (q < 1);
            }
            break;
        case 3:
            if (r <= sml) {
                *W = 495. / (32. * M_PI * sml * sml * sml) * (1 - q) * (1 - q) * (1 - q) * (1 - q) * (1 - q) *
                     (1 - q) * (1. + 6. * q + 35. / 3. * q * q) * (q < 1);
                *dWdr = -1485. / (16. * M_PI * sml * sml * sml * sml) * (1 - q) * (1 - q) * (1 - q) * (1 - q) *
                        (1 - q) * (1. - 35. * q * q + 105. * q * q * q) * (q < 1);
            }
            break;
        default:
            if (r <= sml) {
                *W = 1365. / (64. * M_PI * sml * sml * sml) * (1 - q) * (1 - q) * (1 - q) * (1 - q) * (1 - q) *
                     (1 - q) * (1 - q) * (1 - q) * (1. + 8. * q + 25. * q * q + 32 * q * q * q) * (q < 1);
                *dWdr = -15015. / (32. * M_PI * sml * sml * sml * sml) * q * (1 - q) * (1 - q) * (1 - q) *
                        (1 - q) * (1 - q) * (1 - q) * (1 - q) * (1. + 7 * q + 16 * q * q) * (q < 1);
            }
            break;
    }
    for (int d = 0; d < 3; ++d) dWdx[d] = *dWdr / r * dx[d];
}

// SPH::Kernel::calculateDensity (density.cu:8-72) over a CSR neighbour list;
// avg_h selects h_bar = (h_i + h_j)/2 (VARIABLE_SML || INTEGRATE_SML).
void orc_density(const double* x, const double* y, const double* z, const double* mass,
                 const double* h, int n, const long* off, const int* nbr, int avg_h, int kernel, double* rho) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double W, dWdx[3], dWdr, dx[3] = {0, 0, 0};
        skern(kernel, &W, dWdx, &dWdr, dx, h[i]);
        double r = mass[i] * W;
        for (long k = off[i]; k < off[i + 1]; ++k) {
            int j = nbr[k];
            double sml = avg_h ? 0.5 * (h[i] + h[j]) : h[i];
            dx[0] = x[i] - x[j]; dx[1] = y[i] - y[j]; dx[2] = z[i] - z[j];
            skern(kernel, &W, dWdx, &dWdr, dx, sml);
            r += mass[j] * W;
        }
        rho[i] = r;
    }
}

// SPH::Kernel::calculateSoundSpeed (soundspeed.cu:38-97) followed by
// SPH::Kernel::calculatePressure (pressure.cu:5-87), in the reference's order
// (sound speed first, so the ideal-gas c_s uses the previous pressure).
// eos: 0 polytropic, 1 Murnaghan, 3 isothermal H2, 9 ideal gas,
// 12 locally isothermal.  par = {K, gamma, rho_0, bulk_modulus, n, si_units}.
// Murnaghan and isothermal keep the constant sound speed that
// SPH::Kernel::initializeSoundSpeed (soundspeed.cu:4-36) sets once:
// sqrt(bulk_modulus / rho_0), and 203 m/s (divided by c = 2.998e8 without SI
// units).
void orc_eos(int n, int eos, const double* par, const double* rho, const double* e, double* p,
             double* cs) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        switch (eos) {
            case 0: cs[i] = std::sqrt(par[0] * std::pow(rho[i], par[1] - 1.0)); break;
            case 1: cs[i] = std::sqrt(par[3] / par[2]); break;
            case 3: cs[i] = par[5] != 0.0 ? 203.0 : 203.0 / 2.998e8; break;
            case 9: cs[i] = std::sqrt(par[1] * p[i] / rho[i]); break;
            case 12: cs[i] = 0; break;
            default: break;
        }
        switch (eos) {
            case 0: p[i] = par[0] * std::pow(rho[i], par[1]); break;
            case 1: p[i] = (par[3] / par[4]) * (std::pow(rho[i] / par[2], par[4]) - 1.0); break;
            case 3: p[i] = 41255.407 * rho[i]; break;
            case 9: p[i] = (par[1] - 1) * rho[i] * e[i]; break;
            case 12: p[i] = cs[i] * cs[i] * rho[i]; break;
            default: break;
        }
    }
}

// SPH::Kernel::internalForces, hydro part with SPH_EQU_VERSION 1 and
// Monaghan viscosity (internal_forces.cu:372-552): pressure acceleration
// -m_j (p_i/rho_i^2 + p_j/rho_j^2) gradW, Pi_ij = (beta mu - alpha cbar) mu /
// rhobar for v.r < 0 with mu = hbar v.r/(r^2 + 0.01 hbar^2); drho/dt, de/dt
// (integrate_energy), dh/dt (integrate_sml).
// Balsara switch, SPH::Kernel::CalcDivvandCurlv (kernel.cu:223-342) and the
// factor of internalForces (internal_forces.cu:210-217):
//   div v_i  = sum_j m_j / rho_j (v_j - v_i) . grad W_ij
//   curl v_i = sum_j m_j / rho_i (v_i - v_j) x grad W_ij
//   f_i = |div v_i| / (|div v_i| + |curl v_i| + 1e-4 c_s,i / h_i)
// with grad W at h_i, or at (h_i + h_j)/2 under VARIABLE_SML (avg_h; the
// reference does not average here for INTEGRATE_SML alone).  divv, curlv
// (3 per particle) and f may be null.
void orc_balsara(const double* x, const double* y, const double* z, const double* vx, const double* vy,
                 const double* vz, const double* mass, const double* h, const double* rho, const double* cs,
                 int n, const long* off, const int* nbr, int avg_h, int kernel, double* divv_out,
                 double* curlv_out, double* f) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double divv = 0, curl[3] = {0, 0, 0};
        for (long k = off[i]; k < off[i + 1]; ++k) {
            const int j = nbr[k];
            const double sml = avg_h ? 0.5 * (h[i] + h[j]) : h[i];
            const double dr[3] = {x[i] - x[j], y[i] - y[j], z[i] - z[j]};
            double W, dW[3], dWdr;
            skern(kernel, &W, dW, &dWdr, dr, sml);
            const double vi[3] = {vx[i], vy[i], vz[i]}, vj[3] = {vx[j], vy[j], vz[j]};
            for (int d = 0; d < 3; ++d) divv += mass[j] / rho[j] * (vj[d] - vi[d]) * dW[d];
            curl[0] += mass[j] / rho[i] * ((vi[1] - vj[1]) * dW[2] - (vi[2] - vj[2]) * dW[1]);
            curl[1] += mass[j] / rho[i] * ((vi[2] - vj[2]) * dW[0] - (vi[0] - vj[0]) * dW[2]);
            curl[2] += mass[j] / rho[i] * ((vi[0] - vj[0]) * dW[1] - (vi[1] - vj[1]) * dW[0]);
        }
        if (divv_out) divv_out[i] = divv;
        if (curlv_out) for (int d = 0; d < 3; ++d) curlv_out[3 * (size_t)i + d] = curl[d];
        const double c = std::sqrt(curl[0] * curl[0] + curl[1] * curl[1] + curl[2] * curl[2]);
        if (f) f[i] = std::fabs(divv) / (std::fabs(divv) + c + 1e-4 * cs[i] / h[i]);
    }
}

// bal (may be null): Balsara factors f; the viscous mu_ij is scaled by
// (f_i + f_j)/2 (internal_forces.cu:387-395).
void orc_forces(const double* x, const double* y, const double* z, const double* vx,
                const double* vy, const double* vz, const double* mass, const double* h,
                const double* rho, const double* p, const double* cs, int n, const long* off,
                const int* nbr, double alpha, double beta, int avg_h, int integrate_energy,
                int integrate_sml, int kernel, double* ax, double* ay, double* az, double* drhodt,
                double* dedt, double* dsmldt, const double* bal) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        double acc[3] = {0, 0, 0}, drho = 0, de = 0, dh = 0;
        for (long k = off[i]; k < off[i + 1]; ++k) {
            int j = nbr[k];
            double sml = avg_h ? 0.5 * (h[i] + h[j]) : h[i];
            double dr[3] = {x[i] - x[j], y[i] - y[j], z[i] - z[j]};
            double W, dWdx[3], dWdr;
            skern(kernel, &W, dWdx, &dWdr, dr, sml);
            double dv[3] = {vx[i] - vx[j], vy[i] - vy[j], vz[i] - vz[j]};
            double vvnablaW = dv[0] * dWdx[0] + dv[1] * dWdx[1] + dv[2] * dWdx[2];
            double rr = 0, vr = 0;
            for (int e = 0; e < 3; ++e) { rr += dr[e] * dr[e]; vr += dv[e] * dr[e]; }
            double pij = 0;
            if (vr < 0) {
                double csbar = 0.5 * (cs[i] + cs[j]);
                double smooth = 0.5 * (h[i] + h[j]);
                double mu = smooth * vr / (rr + smooth * smooth * 1e-2);
                double rhobar = 0.5 * (rho[i] + rho[j]);
                if (bal) mu *= (bal[i] + bal[j]) / 2.;
                pij = (beta * mu - alpha * csbar) * mu / rhobar;
            }
            double accj[3];
            for (int d = 0; d < 3; ++d) {
                accj[d] = -mass[j] * (p[i] / (rho[i] * rho[i]) + p[j] / (rho[j] * rho[j])) * dWdx[d];
                acc[d] += accj[d];
            }
            for (int d = 0; d < 3; ++d) acc[d] += mass[j] * (-pij) * dWdx[d];
            drho += rho[i] / rho[j] * mass[j] * vvnablaW;
            if (integrate_sml) dh -= 1. / 3. * h[i] * mass[j] / rho[j] * vvnablaW;
            if (integrate_energy) {
                de += 0.5 * mass[j] * pij * vvnablaW;
                de += 0.5 * accj[0] * -dv[0] + 0.5 * accj[1] * -dv[1] + 0.5 * accj[2] * -dv[2];
            }
        }
        ax[i] = acc[0]; ay[i] = acc[1]; az[i] = acc[2];
        drhodt[i] = drho;
        if (dedt) dedt[i] = integrate_energy ? de : 0.0;
        if (dsmldt) dsmldt[i] = integrate_sml ? dh : 0.0;
    }
}

// Variable smoothing length, SPH::fixedRadiusNN_variableSML (sph.cu:739-961)
// in Jacobi form: in each sweep every unconverged particle counts neighbours
// with d^2 < htmp_i^2 and d^2 < h_j^2 using h_j from the previous sweep (the
// reference reads h_j while other threads overwrite it).  A particle stops
// when nit > 5 or |n - target| < tol, provided n < max_nb; otherwise
// htmp *= 0.5 (1 + (target/n)^{1/3}).  Returns the number of sweeps; h is
// updated in place, counts[] receives the last count.
int orc_variable_h(const double* x, const double* y, const double* z, double* h, int n, int target,
                   int tol, int max_nb, int max_iter, int* counts, double hcap) {
    std::vector<double> hold(h, h + n), hnew(h, h + n);
    std::vector<int> done(n, 0), nit(n, -1);
    std::vector<long> off(n + 1);
    int sweeps = 0;
    for (;;) {
        int active = 0;
        for (int i = 0; i < n; ++i) active += !done[i];
        if (!active) break;
        ++sweeps;
        // counts with d^2 < htmp_i^2 && d^2 < hold_j^2: use a combined radius
        std::vector<int> cnt(n, 0);
        {
            // brute force through the grid: reuse orc_frnn on max(h) radii and filter
            std::vector<double> hr(n);
            for (int i = 0; i < n; ++i) hr[i] = std::max(hnew[i], hold[i]);
            std::vector<long> o(n + 1);
            orc_frnn(x, y, z, hr.data(), n, o.data(), nullptr);
            std::vector<int> nb(o[n]);
            orc_frnn(x, y, z, hr.data(), n, o.data(), nb.data());
#pragma omp parallel for schedule(static)
            for (int i = 0; i < n; ++i) {
                if (done[i]) continue;
                int k = 0;
                for (long q = o[i]; q < o[i + 1]; ++q) {
                    int j = nb[q];
                    double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
                    double d = dx * dx + dy * dy + dz * dz;
                    if (d < hnew[i] * hnew[i] && d < hold[j] * hold[j]) ++k;
                }
                cnt[i] = k;
            }
        }
        for (int i = 0; i < n; ++i) {
            if (done[i]) continue;
            nit[i]++;
            int k = cnt[i];
            counts[i] = k;
            if ((nit[i] > max_iter || std::abs(k - target) < tol) && k < max_nb) {
                done[i] = 1;
            } else {
                int kk = k < 1 ? 1 : k;
                // never past hcap (the edge of the cubic bounding box) when growing
                const double h0 = hnew[i];
                hnew[i] = std::min(h0 * (0.5 * (1.0 + std::pow((double)target / (double)kk, 1. / 3.))),
                                   std::max(hcap, h0));
            }
        }
        hold = hnew;
        if (sweeps > 64) break;
    }
    for (int i = 0; i < n; ++i) h[i] = hnew[i];
    return sweeps;
}

// Neighbour-band repair of this library (no counterpart in the reference,
// whose variable-h iteration, src/sph/sph.cu:739-961, leaves particles whose
// count drifted out of |n - target| < tol after they stopped, or that hit the
// iteration limit, where they are).  Up to `rounds` times: counts with the
// pair rule d^2 < h_i^2 && d^2 < h_j^2; every out-of-band particle i picks,
// with all other h frozen, the h that gives it `want` neighbours (target +
// tol - 2 from above, target - tol + 2 from below): candidates j != i with
// d^2 < rad^2 and d^2 < h_j^2, rad = h_i from above, 1.5 h_i (2 h_i when the
// count is below half of want) from below; more than 256 candidates shrink
// rad by 0.8 (at most 5 tries, then h stays); more than want candidates give
// the midpoint of the want-th and (want+1)-th smallest distances, fewer give
// rad.  From below, rad is capped at twice the h the particle had before the
// first round: a particle whose neighbours' h do not reach it (d >= h_j, at a
// free surface) cannot gain pairs by its own h alone, and its h must not
// grow without bound; nor past hcap (the edge of the cubic bounding box).
// All picks of a round apply at once.  h is updated in place; returns the
// out-of-band count before the first round.
int orc_band_fixup(const double* x, const double* y, const double* z, double* h, int n, int target, int tol,
                   int rounds, double hcap) {
    const int kCap = 256;
    int before = -1;
    std::vector<long> off(n + 1);
    const std::vector<double> h0(h, h + n);
    for (int r = 0; r < rounds; ++r) {
        orc_frnn(x, y, z, h, n, off.data(), nullptr);
        std::vector<int> out;
        for (int i = 0; i < n; ++i)
            if (std::abs((int)(off[i + 1] - off[i]) - target) >= tol) out.push_back(i);
        if (r == 0) before = (int)out.size();
        if (out.empty()) break;
        std::vector<double> hn(h, h + n);
#pragma omp parallel for schedule(dynamic, 16)
        for (size_t q = 0; q < out.size(); ++q) {
            const int i = out[q];
            const int cnt = (int)(off[i + 1] - off[i]);
            const bool above = cnt >= target + tol;
            const int want = above ? target + tol - 2 : target - tol + 2;
            double rad = above ? h[i] : std::min(std::min(2 * cnt >= want ? 1.5 * h[i] : 2.0 * h[i], 2.0 * h0[i]),
                                                 hcap);
            if (!above && rad <= h[i]) continue;  // at the cap: no pair to gain, h stays
            std::vector<double> c;
            for (int attempt = 0; attempt < 5; ++attempt) {
                c.clear();
                const double rad2 = rad * rad;
                for (int j = 0; j < n; ++j) {
                    if (j == i) continue;
                    const double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
                    const double d = dx * dx + dy * dy + dz * dz;
                    if (d < rad2 && d < h[j] * h[j]) c.push_back(d);
                }
                if ((int)c.size() <= kCap) {
                    if ((int)c.size() > want) {
                        std::sort(c.begin(), c.end());
                        hn[i] = 0.5 * (std::sqrt(c[want - 1]) + std::sqrt(c[want]));
                    } else {
                        hn[i] = rad;
                    }
                    break;
                }
                rad = 0.8 * rad;
            }
        }
        for (int i = 0; i < n; ++i) h[i] = hn[i];
    }
    return before;
}

// ---------------------------------------------------------- integrators ---
// LeapfrogNS::Kernel::updateX / updateV (device_leapfrog.cu:4-58).
void orc_leapfrog_x(int n, double dt, double* x, double* y, double* z, const double* vx,
                    const double* vy, const double* vz, const double* gax, const double* gay,
                    const double* gaz, double* gax_old, double* gay_old, double* gaz_old) {
    for (int i = 0; i < n; ++i) {
        x[i] += dt * (vx[i] + 0.5 * dt * gax[i]); gax_old[i] = gax[i];
        y[i] += dt * (vy[i] + 0.5 * dt * gay[i]); gay_old[i] = gay[i];
        z[i] += dt * (vz[i] + 0.5 * dt * gaz[i]); gaz_old[i] = gaz[i];
    }
}
void orc_leapfrog_v(int n, double dt, double* vx, double* vy, double* vz, const double* gax,
                    const double* gay, const double* gaz, const double* gax_old,
                    const double* gay_old, const double* gaz_old) {
    for (int i = 0; i < n; ++i) {
        vx[i] += 0.5 * dt * (gax[i] + gax_old[i]);
        vy[i] += 0.5 * dt * (gay[i] + gay_old[i]);
        vz[i] += 0.5 * dt * (gaz[i] + gaz_old[i]);
    }
}

// ExplicitEulerNS::Kernel::update (device_explicit_euler.cu:4-54): v += dt
// (a + g), then x += dt v with the new v; rho, e (floored at 1e-50) and h
// from their rates when integrated.  a (SPH) and g (gravity) enter only when
// their physics is on (the reference adds zero arrays otherwise).
void orc_euler(int n, double dt, int gravity, int sph, int int_rho, int int_e, int int_sml, double* x,
               double* y, double* z, double* vx, double* vy, double* vz, const double* ax, const double* ay,
               const double* az, const double* gax, const double* gay, const double* gaz, double* rho,
               const double* drhodt, double* e, const double* dedt, double* sml, const double* dsmldt) {
    for (int i = 0; i < n; ++i) {
        double a[3] = {0, 0, 0};
        if (sph) { a[0] = ax[i]; a[1] = ay[i]; a[2] = az[i]; }
        if (gravity) { a[0] += gax[i]; a[1] += gay[i]; a[2] += gaz[i]; }
        vx[i] += dt * a[0]; vy[i] += dt * a[1]; vz[i] += dt * a[2];
        x[i] += dt * vx[i]; y[i] += dt * vy[i]; z[i] += dt * vz[i];
        if (sph && int_rho) rho[i] = rho[i] + dt * drhodt[i];
        if (sph && int_e) {
            e[i] += dt * dedt[i];
            if (e[i] < 1e-50) e[i] = 1e-50;
        }
        if (sph && int_sml) sml[i] = sml[i] + dt * dsmldt[i];
    }
}

int orc_num_threads() { return omp_get_max_threads(); }

}  // extern "C"

extern "C" void orc_gravity_boxes_mono(const double* x, const double* y, const double* z, const double* mass,
                                       const double* q, const int* child, const int* level, const int* sorted,
                                       int n, int gsize, int nsub, double radius, double theta, double eps2,
                                       const double* amag, double alpha, double mono_alpha, double* gax,
                                       double* gay, double* gaz, int* ninter, int* nquad) {
    gravity_boxes_impl(x, y, z, mass, q, child, level, sorted, n, gsize, nsub, radius, theta, eps2, nullptr, 0.0,
                       amag, alpha, 3, gax, gay, gaz, ninter, nquad, mono_alpha);
}
