// Octree built from SFC-sorted keys, in depth-first pre-order.
//
// The reference inserts particles one by one with lock-protected atomics
// (TreeNS::Kernel::buildTree, src/subdomain_key_tree/tree.cu:768-1082), which
// numbers nodes in atomic order.  Here the tree is derived from the sorted
// keys: with d[i] the number of leading octal digits shared by keys i and
// i+1, a cell (prefix, level L) exists exactly where at least two particles
// share the L-digit prefix, i.e. for every maximal run of d >= L.  The cells
// that start at sorted position a are levels d[a-1]+1 .. d[a]; followed by
// the leaf of particle a they form the pre-order of the tree, so one exclusive
// scan of (cells(a) + 1) numbers all nodes.  A node's first child is node+1;
// its subtree ends at `skip`, which makes every walk stackless.
#pragma once
#include "common.cuh"

// info word of nd_link.y: bits 0-7 level, bit 8 leaf flag
#define ND_LEAF 0x100

struct TreeDev {
    int n;              // particles
    int cap_nodes;      // node pool (particles + cells)
    unsigned char* dl;  // [n] common digits of sorted keys a, a+1 (dl[n-1] = 0)
    int* cnt;           // [n] nodes starting at sorted position a
    int* off;           // [n+1] exclusive scan of cnt, off[n] = nodes
    int* leaf_node;     // [n] node id of sorted particle a
    int2* link;         // [cap] (skip, level | ND_LEAF)
    int* first;         // [cap] first sorted particle of the node
    int* last;          // [cap] last sorted particle of the node
    int* parent;        // [cap] parent node, -1 for root children
    int* kids;          // [cap * 8] children by key digit (valid where kmask has the bit)
    int* kmask;         // [cap] bit d: slot d used; 0x100: children without a digit (shared keys)
    double4* com;       // [cap] centre of mass (x, y, z, m)
    float4* bmin;       // [cap] particle bounding box min (rounded down)
    float4* bmax;       // [cap] particle bounding box max (rounded up)
    // [4 * cap] mixed-path walk record, one 64-byte line per node:
    //   [0] float(x), float(y), float(z), m   (FP32 hi part of the centre of mass)
    //   [1] x - float(x), ..., opening criterion edge^2/theta (-1 for leaves)
    //   [2] Qxx Qxy Qxz Qyy  (traceless quadrupole about the centre of mass; 0 for leaves)
    //   [3] Qyz Qzz, bits (link info & 0x1ff) | kmask << 9, M l^3 (cells; l = edge)
    float4* wrec;
    float* hmax;        // [cap] largest smoothing length below the node (rounded up)
    int* arrive;        // [cap] completed children counted for cells that cross a block's
                        // range in the upward pass (0 between passes)
    int* nodes;         // [1] total nodes (= off[n]), device copy
};

int tree_build(TreeDev& T, const uint64_t* skey, void* scan_scratch, DevStatus* st, cudaStream_t s);
// Centres of mass (FP64), quadrupoles and walk records (want_quad, mixed
// walk: every node's wrec, whose geometric criterion uses theta and the root
// edge from the device bounding box `ord`) and particle bounding boxes
// (want_box, used by the neighbour search) of every cell, in one launch.
int tree_upward(TreeDev& T, const double* sx, const double* sy, const double* sz, const double* sm,
                int want_quad, int want_box, const long long* ord, double theta, DevStatus* st, cudaStream_t s);
// T.hmax[node] = max h over the node's particles (h sorted, n entries).
int tree_node_hmax(const TreeDev& T, const double* h, const DevStatus* st, cudaStream_t s);
