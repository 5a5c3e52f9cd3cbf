// Barnes-Hut tangent-point energy: the hierarchical path for curves far larger
// than the dense O(E^2) kernels serve.
//
// The algorithm is the reference's stage-2 oracle (oracle/tpe_stage2_oracle.py):
// an edge bounding-volume tree (build_edge_bvh, :467-502) and a per-target-edge
// traversal (bh_energy, :532-589) with its admissibility rule (:556-557): a
// node of at least two edges, none of which shares a vertex with the target
// edge I, whose spatial radius over the distance from I's midpoint is at most
// theta and whose tangent radius is at most theta_t (default 1.5 theta). An
// admissible node replaces its edges by one source point at its mass-weighted
// center (bh_ordered_cluster_term, :515-529); a leaf that is not admissible is
// summed exactly. theta = 0 admits nothing and gives the exact energy.
//
// The tree is built on the host, in the oracle's order of operations, so that
// the device traverses the same tree: split on the coordinate of largest
// spread of the 6-D points (midpoint, unit tangent), stable sort, the first
// half (rounded down) to the left; node centers, tangents and masses summed as
// numpy sums them (sequential along the rows, pairwise for the mass). Node
// edges are stored as one contiguous range of a permutation of the edges, so
// "does node n contain edge J" is a range test on J's position. The device
// walks the tree once per target edge (one thread each, explicit stack) and
// writes that edge's sum and counts; the totals are reduced in a fixed order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>
#include <utility>
#include <vector>

#include "tpe_internal.h"

namespace tpe {
namespace {

constexpr double kTangentTol = 1e-14;  // TANGENT_TOL of the stage-2 oracle (:34)
constexpr int kStack = 64;             // traversal depth bound (a median tree of 2^31 edges is 32 deep)

struct Node {
    double cx, cy, cz;  // mass-weighted center of the node's edge midpoints
    double mass;        // sum of ell_eps over the node's edges
    double rx, rT;      // max distance of a midpoint (unit tangent) from the center (mean tangent)
    double tx, ty, tz;  // mass-weighted mean of the unit tangents
    int32_t begin, count;  // the node's edges: perm[begin .. begin + count)
    int32_t left, right;   // children, -1 for a leaf
    int32_t parent, pad;
};

// numpy's pairwise summation of a contiguous float64 array (np.sum).
double np_pairwise_sum(const double* a, size_t n) {
    if (n < 8) {
        double s = 0.0;
        for (size_t i = 0; i < n; i++) s += a[i];
        return s;
    }
    if (n <= 128) {
        double r[8];
        for (int j = 0; j < 8; j++) r[j] = a[j];
        size_t i = 8;
        for (; i < n - (n % 8); i += 8)
            for (int j = 0; j < 8; j++) r[j] += a[i + j];
        double res = ((r[0] + r[1]) + (r[2] + r[3])) + ((r[4] + r[5]) + (r[6] + r[7]));
        for (; i < n; i++) res += a[i];
        return res;
    }
    size_t n2 = n / 2;
    n2 -= n2 % 8;
    return np_pairwise_sum(a, n2) + np_pairwise_sum(a + n2, n - n2);
}

inline double norm3(double x, double y, double z) { return std::sqrt((x * x + y * y) + z * z); }

using Keyed = std::vector<std::pair<double, int32_t>>;

// std::stable_sort on the key, with the range cut into up to `threads` pieces
// sorted on their own threads and merged pairwise (std::merge takes from the
// first range on ties, so the order is the same stable order).
void stable_sort_keys(Keyed& a, int threads) {
    auto less = [](const std::pair<double, int32_t>& x, const std::pair<double, int32_t>& y) {
        return x.first < y.first;
    };
    const size_t n = a.size();
    int p = 1;
    while (p * 2 <= threads && n / (size_t)(p * 2) >= 16384) p *= 2;
    if (p == 1) {
        std::stable_sort(a.begin(), a.end(), less);
        return;
    }
    std::vector<size_t> cut((size_t)p + 1);
    for (int i = 0; i <= p; i++) cut[i] = n * (size_t)i / (size_t)p;
    auto run = [&](std::vector<std::thread>& th, auto&& body, int count) {
        try {
            for (int i = 0; i < count; i++) th.emplace_back(body, i);
        } catch (...) {
            for (auto& t : th) t.join();
            throw;
        }
        for (auto& t : th) t.join();
    };
    {
        std::vector<std::thread> th;
        run(th, [&](int i) { std::stable_sort(a.begin() + cut[i], a.begin() + cut[i + 1], less); }, p);
    }
    Keyed b(n);
    for (int w = 1; w < p; w *= 2) {
        std::vector<std::thread> th;
        const int pairs = p / (2 * w);
        run(th,
            [&](int j) {
                const size_t lo = cut[2 * w * j], mid = cut[2 * w * j + w], hi = cut[2 * w * (j + 1)];
                std::merge(a.begin() + lo, a.begin() + mid, a.begin() + mid, a.begin() + hi,
                           b.begin() + lo, less);
            },
            pairs);
        a.swap(b);
    }
}

struct Builder {
    const std::vector<double>& C;  // E x 3 midpoints
    const std::vector<double>& T;  // E x 3 unit tangents
    const std::vector<double>& m;  // E masses (ell_eps)
    int32_t leaf;
    int32_t* perm;                 // shared; a builder writes only its own ranges
    std::vector<Node> nodes;
    std::vector<double> tmp;
    Keyed keyed;
    int sort_threads = 1;  // threads for the sort of one node (the top levels)
    // subtrees at depth split_depth are left to other builders: (begin, count,
    // parent node, is-left) each, the parent's child link holding -2 - task
    int32_t split_depth = -1;
    struct Task {
        int32_t begin, count, parent;
        bool left;
    };
    std::vector<Task> tasks;

    int32_t rec(int32_t begin, int32_t count, int32_t depth = 0) {
        const int32_t* idx = perm + begin;
        tmp.resize((size_t)count);
        for (int32_t k = 0; k < count; k++) tmp[k] = m[idx[k]];
        const double msum = np_pairwise_sum(tmp.data(), (size_t)count);
        double c[3] = {0, 0, 0}, t[3] = {0, 0, 0};
        for (int32_t k = 0; k < count; k++) {
            const int32_t J = idx[k];
            for (int d = 0; d < 3; d++) {
                c[d] = c[d] + m[J] * C[3 * (size_t)J + d];
                t[d] = t[d] + m[J] * T[3 * (size_t)J + d];
            }
        }
        for (int d = 0; d < 3; d++) {
            c[d] = c[d] / msum;
            t[d] = t[d] / msum;
        }
        double rx = 0.0, rT = 0.0;
        for (int32_t k = 0; k < count; k++) {
            const int32_t J = idx[k];
            rx = std::max(rx, norm3(C[3 * (size_t)J] - c[0], C[3 * (size_t)J + 1] - c[1],
                                    C[3 * (size_t)J + 2] - c[2]));
            rT = std::max(rT, norm3(T[3 * (size_t)J] - t[0], T[3 * (size_t)J + 1] - t[1],
                                    T[3 * (size_t)J + 2] - t[2]));
        }
        const int32_t me = (int32_t)nodes.size();
        nodes.push_back(Node{c[0], c[1], c[2], msum, rx, rT, t[0], t[1], t[2], begin, count, -1, -1, -1, 0});
        if (count > leaf) {
            // the coordinate of largest spread (first on ties), stable sort on it
            double lo[6], hi[6];
            for (int d = 0; d < 6; d++) {
                lo[d] = INFINITY;
                hi[d] = -INFINITY;
            }
            for (int32_t k = 0; k < count; k++) {
                const int32_t J = idx[k];
                for (int d = 0; d < 6; d++) {
                    const double x = d < 3 ? C[3 * (size_t)J + d] : T[3 * (size_t)J + d - 3];
                    lo[d] = std::min(lo[d], x);
                    hi[d] = std::max(hi[d], x);
                }
            }
            int dim = 0;
            double best = hi[0] - lo[0];
            for (int d = 1; d < 6; d++)
                if (hi[d] - lo[d] > best) {
                    best = hi[d] - lo[d];
                    dim = d;
                }
            const std::vector<double>& X = dim < 3 ? C : T;
            const int dd = dim % 3;
            keyed.resize((size_t)count);
            for (int32_t k = 0; k < count; k++) keyed[k] = {X[3 * (size_t)idx[k] + dd], idx[k]};
            stable_sort_keys(keyed, sort_threads);
            for (int32_t k = 0; k < count; k++) perm[begin + k] = keyed[k].second;
            const int32_t mid = count / 2;
            int32_t l, r;
            if (depth + 1 == split_depth) {
                tasks.push_back({begin, mid, me, true});
                l = -2 - (int32_t)(tasks.size() - 1);
                tasks.push_back({begin + mid, count - mid, me, false});
                r = -2 - (int32_t)(tasks.size() - 1);
            } else {
                l = rec(begin, mid, depth + 1);
                r = rec(begin + mid, count - mid, depth + 1);
                nodes[l].parent = me;
                nodes[r].parent = me;
            }
            nodes[me].left = l;
            nodes[me].right = r;
        }
        return me;
    }
};

__device__ __forceinline__ double term(double ex, double ey, double ez, double dx, double dy,
                                       double dz, double alpha, double beta, double eps) {
    const double cx = ey * dz - ez * dy, cy = ez * dx - ex * dz, cz = ex * dy - ey * dx;
    const double dn = sqrt((dx * dx + dy * dy) + dz * dz) + eps;
    const double cn = sqrt((cx * cx + cy * cy) + cz * cz) + eps;
    return pow(cn, alpha) / pow(dn, beta);
}

// One thread per target edge I: its ordered sum over the tree, and the visit,
// approximated-edge and direct-pair counts.
__global__ void __launch_bounds__(128)
bh_energy_kernel(const double* __restrict__ pos, const int2* __restrict__ edges, int32_t E,
                 const Node* __restrict__ nodes, const int32_t* __restrict__ perm,
                 const int32_t* __restrict__ where, const int32_t* __restrict__ inc_off,
                 const int32_t* __restrict__ inc, double alpha, double beta, double eps,
                 double theta, double theta_t, double* __restrict__ out,
                 long long* __restrict__ counts, int32_t* __restrict__ err) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= E) return;
    const int2 eI = edges[I];
    const double ax = pos[3 * eI.x], ay = pos[3 * eI.x + 1], az = pos[3 * eI.x + 2];
    const double bx = pos[3 * eI.y], by = pos[3 * eI.y + 1], bz = pos[3 * eI.y + 2];
    const double ex = bx - ax, ey = by - ay, ez = bz - az;
    const double ellI = sqrt((ex * ex + ey * ey) + ez * ez) + eps;
    const double pI = pow(ellI, 1.0 - alpha);
    const double mx = 0.5 * (ax + bx), my = 0.5 * (ay + by), mz = 0.5 * (az + bz);
    double val = 0.0;
    long long visits = 0, approx = 0, direct = 0;
    int32_t stack[kStack];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const Node nd = nodes[stack[--sp]];
        visits++;
        const double dist = sqrt(((mx - nd.cx) * (mx - nd.cx) + (my - nd.cy) * (my - nd.cy)) +
                                 (mz - nd.cz) * (mz - nd.cz));
        bool admiss = nd.count >= 2 && dist > 0.0 && nd.rx / dist <= theta && nd.rT <= theta_t;
        if (admiss) {
            // no edge of the node may share a vertex with I (I itself included)
            for (int s = 0; s < 2 && admiss; s++) {
                const int32_t v = s ? eI.y : eI.x;
                for (int32_t q = inc_off[v]; q < inc_off[v + 1]; q++) {
                    const int32_t w = where[inc[q] >> 1];
                    if (w >= nd.begin && w < nd.begin + nd.count) {
                        admiss = false;
                        break;
                    }
                }
            }
        }
        if (admiss) {
            approx += nd.count;
            const double s = term(ex, ey, ez, ax - nd.cx, ay - nd.cy, az - nd.cz, alpha, beta, eps) +
                             term(ex, ey, ez, bx - nd.cx, by - nd.cy, bz - nd.cz, alpha, beta, eps);
            val += 0.5 * pI * nd.mass * s;
        } else if (nd.left < 0) {
            for (int32_t k = nd.begin; k < nd.begin + nd.count; k++) {
                const int32_t J = perm[k];
                const int2 eJ = edges[J];
                if (J == I || eJ.x == eI.x || eJ.x == eI.y || eJ.y == eI.x || eJ.y == eI.y) continue;
                direct++;
                const double cx = pos[3 * eJ.x], cy = pos[3 * eJ.x + 1], cz = pos[3 * eJ.x + 2];
                const double dx = pos[3 * eJ.y], dy = pos[3 * eJ.y + 1], dz = pos[3 * eJ.y + 2];
                const double fx = dx - cx, fy = dy - cy, fz = dz - cz;
                const double ellJ = sqrt((fx * fx + fy * fy) + fz * fz) + eps;
                const double s = term(ex, ey, ez, ax - cx, ay - cy, az - cz, alpha, beta, eps) +
                                 term(ex, ey, ez, ax - dx, ay - dy, az - dz, alpha, beta, eps) +
                                 term(ex, ey, ez, bx - cx, by - cy, bz - cz, alpha, beta, eps) +
                                 term(ex, ey, ez, bx - dx, by - dy, bz - dz, alpha, beta, eps);
                val += 0.25 * pI * ellJ * s;
            }
        } else {
            if (sp + 2 > kStack) {
                atomicExch(err, 1);
                break;
            }
            stack[sp++] = nd.right;
            stack[sp++] = nd.left;
        }
    }
    out[I] = val;
    counts[3 * (size_t)I] = visits;
    counts[3 * (size_t)I + 1] = approx;
    counts[3 * (size_t)I + 2] = direct;
}

// Fixed-order totals: one block sums the per-edge values and counts.
__global__ void __launch_bounds__(256)
bh_reduce_kernel(const double* __restrict__ val, const long long* __restrict__ counts, int32_t E,
                 double* __restrict__ total, long long* __restrict__ ctot) {
    __shared__ double sv[256];
    __shared__ long long sc[3][256];
    double v = 0.0;
    long long c0 = 0, c1 = 0, c2 = 0;
    for (int32_t i = threadIdx.x; i < E; i += 256) {
        v += val[i];
        c0 += counts[3 * (size_t)i];
        c1 += counts[3 * (size_t)i + 1];
        c2 += counts[3 * (size_t)i + 2];
    }
    sv[threadIdx.x] = v;
    sc[0][threadIdx.x] = c0;
    sc[1][threadIdx.x] = c1;
    sc[2][threadIdx.x] = c2;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sv[threadIdx.x] += sv[threadIdx.x + s];
            for (int q = 0; q < 3; q++) sc[q][threadIdx.x] += sc[q][threadIdx.x + s];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        total[0] = 0.5 * sv[0];
        for (int q = 0; q < 3; q++) ctot[q] = sc[q][0];
    }
}

// Edge geometry as edge_geometry computes it (tpe_stage2_oracle.py:72-82) and
// the tree over it.
struct Tree {
    std::vector<double> C, T, m;  // midpoints, unit tangents (E x 3), ell_eps (E)
    std::vector<Node> nodes;
    std::vector<int32_t> perm, where;  // edge at each position, position of each edge
};

void build_tree(const int32_t* edges, int32_t E, const double* h_xyz, double eps, int32_t leaf,
                Tree& tr) {
    tr.C.assign((size_t)3 * E, 0.0);
    tr.T.assign((size_t)3 * E, 0.0);
    tr.m.assign((size_t)E, 0.0);
    for (int32_t I = 0; I < E; I++) {
        const int32_t a = edges[2 * (size_t)I], b = edges[2 * (size_t)I + 1];
        double e[3];
        for (int d = 0; d < 3; d++) {
            e[d] = h_xyz[3 * (size_t)b + d] - h_xyz[3 * (size_t)a + d];
            tr.C[3 * (size_t)I + d] = 0.5 * (h_xyz[3 * (size_t)a + d] + h_xyz[3 * (size_t)b + d]);
        }
        const double ell = norm3(e[0], e[1], e[2]);
        for (int d = 0; d < 3; d++) tr.T[3 * (size_t)I + d] = ell >= kTangentTol ? e[d] / ell : 0.0;
        tr.m[I] = ell + eps;
    }
    tr.perm.resize((size_t)E);
    std::iota(tr.perm.begin(), tr.perm.end(), 0);
    // The top levels on this thread; below them, subtrees on their own threads
    // (disjoint ranges of the permutation, the same arithmetic), then joined.
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    int32_t split = 0;
    while ((1u << split) < std::min(hw, 16u) && ((int64_t)E >> split) > 4 * (int64_t)leaf + 4096) split++;
    Builder top{tr.C, tr.T, tr.m, leaf, tr.perm.data(), {}, {}, {}, 1, split > 0 ? split : -1, {}};
    top.sort_threads = (int)std::min(hw, 16u);
    top.rec(0, E);
    std::vector<Builder> sub;
    sub.reserve(top.tasks.size());
    for (size_t i = 0; i < top.tasks.size(); i++)
        sub.push_back(Builder{tr.C, tr.T, tr.m, leaf, tr.perm.data(), {}, {}, {}, 1, -1, {}});
    {
        // a failure inside a worker (allocation) is carried back to this thread
        std::vector<char> failed(top.tasks.size(), 0);
        std::vector<std::thread> th;
        try {
            for (size_t i = 0; i < top.tasks.size(); i++)
                th.emplace_back([&, i] {
                    try {
                        sub[i].rec(top.tasks[i].begin, top.tasks[i].count);
                    } catch (...) {
                        failed[i] = 1;
                    }
                });
        } catch (...) {
            for (auto& x : th) x.join();
            throw;
        }
        for (auto& x : th) x.join();
        for (char f : failed)
            if (f) throw std::bad_alloc();
    }
    tr.nodes.swap(top.nodes);
    for (size_t i = 0; i < sub.size(); i++) {
        const int32_t base = (int32_t)tr.nodes.size();
        for (Node nd : sub[i].nodes) {
            if (nd.left >= 0) {
                nd.left += base;
                nd.right += base;
            }
            if (nd.parent >= 0) nd.parent += base;
            tr.nodes.push_back(nd);
        }
        const Builder::Task& tk = top.tasks[i];
        tr.nodes[base].parent = tk.parent;
        (tk.left ? tr.nodes[tk.parent].left : tr.nodes[tk.parent].right) = base;
    }
    tr.where.assign((size_t)E, 0);
    for (int32_t k = 0; k < E; k++) tr.where[tr.perm[k]] = k;
}

}  // namespace

int32_t bh_energy(tpe_ctx* ctx, const double* h_xyz, const double* d_xyz, double alpha, double beta,
                  double eps, double theta, double theta_t, int32_t leaf, double* energy,
                  int64_t* stats) {
    const int32_t E = ctx->E;
    if (leaf < 1 || !(theta >= 0.0) || !(theta_t >= 0.0)) {
        set_error(ctx, TPE_ERR_BAD_ARG, "bh energy: leaf size >= 1 and theta, theta_t >= 0");
        return TPE_ERR_BAD_ARG;
    }
    if (E == 0) {
        *energy = 0.0;
        if (stats) stats[0] = stats[1] = stats[2] = 0;
        return TPE_OK;
    }
    Tree tr;
    build_tree(ctx->h_edges.data(), ctx->E, h_xyz, eps, leaf, tr);
    const size_t nn = tr.nodes.size();
    const size_t bytes_nodes = sizeof(Node) * nn, bytes_idx = sizeof(int32_t) * (size_t)E;
    const size_t off_perm = (bytes_nodes + 255) / 256 * 256;
    const size_t off_where = off_perm + (bytes_idx + 255) / 256 * 256;
    const size_t off_val = off_where + (bytes_idx + 255) / 256 * 256;
    const size_t off_cnt = off_val + (sizeof(double) * (size_t)E + 255) / 256 * 256;
    const size_t off_tot = off_cnt + (sizeof(long long) * 3 * (size_t)E + 255) / 256 * 256;
    TPE_TRY(ensure(ctx, ctx->bh_buf, off_tot + 256));
    uint8_t* base = ctx->bh_buf.as<uint8_t>();
    const cudaStream_t st = ctx->stream;
    TPE_CUDA_TRY(cudaMemcpyAsync(base, tr.nodes.data(), bytes_nodes, cudaMemcpyHostToDevice, st));
    TPE_CUDA_TRY(cudaMemcpyAsync(base + off_perm, tr.perm.data(), bytes_idx, cudaMemcpyHostToDevice, st));
    TPE_CUDA_TRY(cudaMemcpyAsync(base + off_where, tr.where.data(), bytes_idx, cudaMemcpyHostToDevice, st));
    int32_t* err = reinterpret_cast<int32_t*>(base + off_tot + 32);
    TPE_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int32_t), st));
    {
        KernelScope ks(ctx, TPE_KGROUP_ENERGY, 2);
        bh_energy_kernel<<<(E + 127) / 128, 128, 0, st>>>(
            d_xyz, ctx->d_edges.as<int2>(), E, reinterpret_cast<const Node*>(base),
            reinterpret_cast<const int32_t*>(base + off_perm),
            reinterpret_cast<const int32_t*>(base + off_where), ctx->d_inc_off.as<int32_t>(),
            ctx->d_inc.as<int32_t>(), alpha, beta, eps, theta, theta_t,
            reinterpret_cast<double*>(base + off_val), reinterpret_cast<long long*>(base + off_cnt), err);
        TPE_CUDA_TRY(cudaGetLastError());
        bh_reduce_kernel<<<1, 256, 0, st>>>(reinterpret_cast<const double*>(base + off_val),
                                            reinterpret_cast<const long long*>(base + off_cnt), E,
                                            reinterpret_cast<double*>(base + off_tot),
                                            reinterpret_cast<long long*>(base + off_tot + 8));
        TPE_CUDA_TRY(cudaGetLastError());
    }
    // total (8 bytes), three counts (24 bytes), the stack flag (4 bytes)
    unsigned char h[36];
    TPE_CUDA_TRY(cudaMemcpyAsync(h, base + off_tot, sizeof(h), cudaMemcpyDeviceToHost, st));
    TPE_CUDA_TRY(cudaStreamSynchronize(st));
    int32_t herr = 0;
    memcpy(&herr, h + 32, sizeof(int32_t));
    if (herr) {
        set_error(ctx, TPE_ERR_INTERNAL, "bh energy: tree deeper than the traversal stack");
        return TPE_ERR_INTERNAL;
    }
    memcpy(energy, h, sizeof(double));
    if (stats) {
        long long c[3];
        memcpy(c, h + 8, sizeof(c));
        for (int q = 0; q < 3; q++) stats[q] = (int64_t)c[q];
    }
    return TPE_OK;
}


// ---- block-cluster-tree kernel products (bct_matvec_kernel) -------------------------
//
// phi = K psi for the high- or low-order edge kernel K of the Sobolev inner
// product, the stage-2 oracle's bct_matvec_kernel (tpe_stage2_oracle.py:649-703):
// a dual traversal of the edge tree from (root, root); a block (t, s) is
// admissible when it holds at least three edges, no edge of t shares a vertex
// with an edge of s, max(rx) / distance <= theta and max(rT) <= theta_t; it then
// adds mass_I * k(t, s) * sum_{J in s} mass_J psi_J to every I in t, with k the
// node kernel (bct_kernel_node :634-643). Two leaves that are not admissible are
// summed pair by pair with the exact edge kernel (exact_edge_kernel_pair
// :706-730). Otherwise the target splits when it is not a leaf and the source is
// a leaf or no larger, else the source splits. The block list is built on the
// host (the same recursion); the device forms every node's moment
// sum_J mass_J psi_J, each target node's sum of k * moment over its admissible
// blocks, and per edge the sum over its tree ancestors plus its direct blocks.

namespace {

struct BctLists {
    std::vector<int32_t> adm_t, adm_s, dir_t, dir_s;
    std::vector<double> adm_k;
    int64_t admissible = 0, direct_blocks = 0, direct_pairs = 0;
};

double node_kernel(int kind, const Node& t, const Node& s, double eps) {
    const double dx = t.cx - s.cx, dy = t.cy - s.cy, dz = t.cz - s.cz;
    const double dn = norm3(dx, dy, dz) + eps;
    if (kind == 0) return 2.0 / std::pow(dn, 7.0 / 3.0);
    // |t_T x d| and |t_S x (-d)|
    const double c1 = norm3(t.ty * dz - t.tz * dy, t.tz * dx - t.tx * dz, t.tx * dy - t.ty * dx) + eps;
    const double c2 = norm3(s.ty * -dz - s.tz * -dy, s.tz * -dx - s.tx * -dz, s.tx * -dy - s.ty * -dx) + eps;
    return (std::pow(c1, 2.0) + std::pow(c2, 2.0)) / std::pow(dn, 4.0 + 7.0 / 3.0);
}

struct BctRec {
    const Tree& tr;
    const tpe_ctx* ctx;
    int kind;
    double eps, theta, theta_t;
    BctLists& out;

    bool shares(int32_t I, int32_t J) const {
        const int32_t* e = ctx->h_edges.data();
        return I == J || e[2 * I] == e[2 * J] || e[2 * I] == e[2 * J + 1] || e[2 * I + 1] == e[2 * J] ||
               e[2 * I + 1] == e[2 * J + 1];
    }
    // no edge of t shares a vertex with an edge of s (blocks_all_disjoint); the
    // relation is symmetric, so the smaller node's edges are looked up in the other
    bool disjoint(const Node& t0, const Node& s0) const {
        const Node& t = t0.count <= s0.count ? t0 : s0;
        const Node& s = t0.count <= s0.count ? s0 : t0;
        for (int32_t k = t.begin; k < t.begin + t.count; k++) {
            const int32_t I = tr.perm[k];
            for (int q = 0; q < 2; q++) {
                const int32_t v = ctx->h_edges[2 * (size_t)I + q];
                for (int32_t r = ctx->h_inc_off[v]; r < ctx->h_inc_off[v + 1]; r++) {
                    const int32_t w = tr.where[ctx->h_inc[r] >> 1];
                    if (w >= s.begin && w < s.begin + s.count) return false;
                }
            }
        }
        return true;
    }
    void rec(int32_t ti, int32_t si) {
        const Node& tn = tr.nodes[ti];
        const Node& sn = tr.nodes[si];
        const double dist = norm3(tn.cx - sn.cx, tn.cy - sn.cy, tn.cz - sn.cz);
        const bool well = tn.count + sn.count >= 3 && dist > 0.0 &&
                          std::max(tn.rx, sn.rx) / dist <= theta && std::max(tn.rT, sn.rT) <= theta_t &&
                          disjoint(tn, sn);
        if (well) {
            out.adm_t.push_back(ti);
            out.adm_s.push_back(si);
            out.adm_k.push_back(node_kernel(kind, tn, sn, eps));
            out.admissible++;
            return;
        }
        if (tn.left < 0 && sn.left < 0) {
            out.dir_t.push_back(ti);
            out.dir_s.push_back(si);
            out.direct_blocks++;
            for (int32_t a = tn.begin; a < tn.begin + tn.count; a++)
                for (int32_t b = sn.begin; b < sn.begin + sn.count; b++)
                    if (!shares(tr.perm[a], tr.perm[b])) out.direct_pairs++;
            return;
        }
        const bool split_t = tn.left >= 0 && (sn.left < 0 || tn.count >= sn.count);
        if (split_t) {
            rec(tn.left, si);
            rec(tn.right, si);
        } else {
            rec(ti, sn.left);
            rec(ti, sn.right);
        }
    }
};

// CSR of (key, value) pairs grouped by key, keeping the recorded order in a group.
void csr(int32_t nkeys, const std::vector<int32_t>& key, std::vector<int32_t>& off,
         std::vector<int32_t>& order) {
    off.assign((size_t)nkeys + 1, 0);
    for (int32_t k : key) off[k + 1]++;
    for (int32_t i = 0; i < nkeys; i++) off[i + 1] += off[i];
    order.assign(key.size(), 0);
    std::vector<int32_t> fill(off.begin(), off.end() - 1);
    for (size_t i = 0; i < key.size(); i++) order[fill[key[i]]++] = (int32_t)i;
}

// moment[n][c] = sum over the node's edges of mass_J psi_J[c]
__global__ void bct_moment_kernel(const Node* __restrict__ nodes, int32_t nn,
                                  const int32_t* __restrict__ perm, const double* __restrict__ mass,
                                  const double* __restrict__ psi, int32_t nr, double* __restrict__ mom) {
    const int32_t n = blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= nn) return;
    const Node nd = nodes[n];
    double acc[3] = {0.0, 0.0, 0.0};
    for (int32_t k = nd.begin; k < nd.begin + nd.count; k++) {
        const int32_t J = perm[k];
        for (int c = 0; c < nr; c++) acc[c] += mass[J] * psi[(size_t)J * nr + c];
    }
    for (int c = 0; c < nr; c++) mom[(size_t)n * nr + c] = acc[c];
}

// local[t][c] = sum over t's admissible blocks (s, k) of k * moment[s][c]
__global__ void bct_local_kernel(int32_t nn, const int32_t* __restrict__ off,
                                 const int32_t* __restrict__ src, const double* __restrict__ kv,
                                 const double* __restrict__ mom, int32_t nr, double* __restrict__ loc) {
    const int32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nn) return;
    double acc[3] = {0.0, 0.0, 0.0};
    for (int32_t b = off[t]; b < off[t + 1]; b++)
        for (int c = 0; c < nr; c++) acc[c] += kv[b] * mom[(size_t)src[b] * nr + c];
    for (int c = 0; c < nr; c++) loc[(size_t)t * nr + c] = acc[c];
}

__device__ __forceinline__ double exact_pair_kernel(int kind, const double* __restrict__ pos, int2 eI,
                                                    int2 eJ, double eps) {
    const double p = 7.0 / 3.0;
    const double ax = pos[3 * eI.x], ay = pos[3 * eI.x + 1], az = pos[3 * eI.x + 2];
    const double bx = pos[3 * eI.y], by = pos[3 * eI.y + 1], bz = pos[3 * eI.y + 2];
    const double cx = pos[3 * eJ.x], cy = pos[3 * eJ.x + 1], cz = pos[3 * eJ.x + 2];
    const double dx = pos[3 * eJ.y], dy = pos[3 * eJ.y + 1], dz = pos[3 * eJ.y + 2];
    const double ux = bx - ax, uy = by - ay, uz = bz - az, wx = dx - cx, wy = dy - cy, wz = dz - cz;
    const double lI = sqrt((ux * ux + uy * uy) + uz * uz), lJ = sqrt((wx * wx + wy * wy) + wz * wz);
    const double ellI = lI + eps, ellJ = lJ + eps;
    double tI[3] = {0, 0, 0}, tJ[3] = {0, 0, 0};
    if (lI >= kTangentTol) {
        tI[0] = ux / lI;
        tI[1] = uy / lI;
        tI[2] = uz / lI;
    }
    if (lJ >= kTangentTol) {
        tJ[0] = wx / lJ;
        tJ[1] = wy / lJ;
        tJ[2] = wz / lJ;
    }
    const double vi[2][3] = {{ax, ay, az}, {bx, by, bz}}, vj[2][3] = {{cx, cy, cz}, {dx, dy, dz}};
    double s1 = 0.0, s2 = 0.0;
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            const double qx = vi[i][0] - vj[j][0], qy = vi[i][1] - vj[j][1], qz = vi[i][2] - vj[j][2];
            const double dn = sqrt((qx * qx + qy * qy) + qz * qz) + eps;
            if (kind == 0) {
                s1 += 1.0 / pow(dn, p);
            } else {
                const double c1 = sqrt(((tI[1] * qz - tI[2] * qy) * (tI[1] * qz - tI[2] * qy) +
                                        (tI[2] * qx - tI[0] * qz) * (tI[2] * qx - tI[0] * qz)) +
                                       (tI[0] * qy - tI[1] * qx) * (tI[0] * qy - tI[1] * qx)) + eps;
                const double c2 = sqrt(((tJ[1] * -qz - tJ[2] * -qy) * (tJ[1] * -qz - tJ[2] * -qy) +
                                        (tJ[2] * -qx - tJ[0] * -qz) * (tJ[2] * -qx - tJ[0] * -qz)) +
                                       (tJ[0] * -qy - tJ[1] * -qx) * (tJ[0] * -qy - tJ[1] * -qx)) + eps;
                const double den = pow(dn, 4.0 + p);
                s1 += pow(c1, 2.0) / den;
                s2 += pow(c2, 2.0) / den;
            }
        }
    return kind == 0 ? 2.0 * 0.25 * ellI * ellJ * s1 : 0.25 * ellI * ellJ * (s1 + s2);
}

// per edge I: mass_I times the ancestors' local sums, plus its leaf's direct blocks
__global__ void bct_apply_kernel(int kind, const double* __restrict__ pos, const int2* __restrict__ edges,
                                 int32_t E, const Node* __restrict__ nodes,
                                 const int32_t* __restrict__ perm, const int32_t* __restrict__ leaf_of,
                                 const double* __restrict__ mass, const double* __restrict__ loc,
                                 const int32_t* __restrict__ doff, const int32_t* __restrict__ dsrc,
                                 const double* __restrict__ psi, int32_t nr, double eps,
                                 double* __restrict__ phi) {
    const int32_t I = blockIdx.x * blockDim.x + threadIdx.x;
    if (I >= E) return;
    const int32_t leaf = leaf_of[I];
    double far[3] = {0.0, 0.0, 0.0}, near[3] = {0.0, 0.0, 0.0};
    for (int32_t n = leaf; n >= 0; n = nodes[n].parent)
        for (int c = 0; c < nr; c++) far[c] += loc[(size_t)n * nr + c];
    const int2 eI = edges[I];
    for (int32_t b = doff[leaf]; b < doff[leaf + 1]; b++) {
        const Node sn = nodes[dsrc[b]];
        for (int32_t k = sn.begin; k < sn.begin + sn.count; k++) {
            const int32_t J = perm[k];
            const int2 eJ = edges[J];
            if (J == I || eJ.x == eI.x || eJ.x == eI.y || eJ.y == eI.x || eJ.y == eI.y) continue;
            const double kij = exact_pair_kernel(kind, pos, eI, eJ, eps);
            for (int c = 0; c < nr; c++) near[c] += kij * psi[(size_t)J * nr + c];
        }
    }
    for (int c = 0; c < nr; c++) phi[(size_t)I * nr + c] = mass[I] * far[c] + near[c];
}

}  // namespace

int32_t bct_matvec(tpe_ctx* ctx, const double* h_xyz, const double* d_xyz, int32_t kind,
                   const double* h_psi, int32_t nr, double eps, double theta, double theta_t,
                   int32_t leaf, double* h_phi, int64_t* stats) {
    const int32_t E = ctx->E;
    if (leaf < 1 || !(theta >= 0.0) || !(theta_t >= 0.0) || (kind != 0 && kind != 1) ||
        (nr != 1 && nr != 3)) {
        set_error(ctx, TPE_ERR_BAD_ARG, "bct matvec: kind 0/1, 1 or 3 columns, leaf >= 1, theta >= 0");
        return TPE_ERR_BAD_ARG;
    }
    if (E == 0) {
        if (stats) stats[0] = stats[1] = stats[2] = stats[3] = 0;
        return TPE_OK;
    }
    Tree tr;
    build_tree(ctx->h_edges.data(), ctx->E, h_xyz, eps, leaf, tr);
    BctLists L;
    BctRec R{tr, ctx, kind, eps, theta, theta_t, L};
    R.rec(0, 0);
    const int32_t nn = (int32_t)tr.nodes.size();
    std::vector<int32_t> aoff, aord, doff, dord;
    csr(nn, L.adm_t, aoff, aord);
    csr(nn, L.dir_t, doff, dord);
    std::vector<int32_t> asrc(aord.size()), dsrc(dord.size());
    std::vector<double> akv(aord.size());
    for (size_t i = 0; i < aord.size(); i++) {
        asrc[i] = L.adm_s[aord[i]];
        akv[i] = L.adm_k[aord[i]];
    }
    for (size_t i = 0; i < dord.size(); i++) dsrc[i] = L.dir_s[dord[i]];
    std::vector<int32_t> leaf_of((size_t)E, 0);
    for (int32_t n = 0; n < nn; n++)
        if (tr.nodes[n].left < 0)
            for (int32_t k = tr.nodes[n].begin; k < tr.nodes[n].begin + tr.nodes[n].count; k++)
                leaf_of[tr.perm[k]] = n;
    // device layout, 256-byte aligned pieces
    size_t off = 0;
    auto piece = [&](size_t bytes) {
        const size_t o = off;
        off += (bytes + 255) / 256 * 256;
        return o;
    };
    const size_t o_nodes = piece(sizeof(Node) * nn), o_perm = piece(sizeof(int32_t) * E),
                 o_leaf = piece(sizeof(int32_t) * E), o_mass = piece(sizeof(double) * E),
                 o_aoff = piece(sizeof(int32_t) * (nn + 1)), o_asrc = piece(sizeof(int32_t) * (asrc.size() + 1)),
                 o_akv = piece(sizeof(double) * (akv.size() + 1)), o_doff = piece(sizeof(int32_t) * (nn + 1)),
                 o_dsrc = piece(sizeof(int32_t) * (dsrc.size() + 1)), o_psi = piece(sizeof(double) * E * nr),
                 o_mom = piece(sizeof(double) * nn * nr), o_loc = piece(sizeof(double) * nn * nr),
                 o_phi = piece(sizeof(double) * E * nr);
    TPE_TRY(ensure(ctx, ctx->bh_buf, off));
    uint8_t* base = ctx->bh_buf.as<uint8_t>();
    const cudaStream_t st = ctx->stream;
    auto up = [&](size_t o, const void* h, size_t bytes) -> int32_t {
        if (bytes) TPE_CUDA_TRY(cudaMemcpyAsync(base + o, h, bytes, cudaMemcpyHostToDevice, st));
        return TPE_OK;
    };
    TPE_TRY(up(o_nodes, tr.nodes.data(), sizeof(Node) * nn));
    TPE_TRY(up(o_perm, tr.perm.data(), sizeof(int32_t) * E));
    TPE_TRY(up(o_leaf, leaf_of.data(), sizeof(int32_t) * E));
    TPE_TRY(up(o_mass, tr.m.data(), sizeof(double) * E));
    TPE_TRY(up(o_aoff, aoff.data(), sizeof(int32_t) * (nn + 1)));
    TPE_TRY(up(o_asrc, asrc.data(), sizeof(int32_t) * asrc.size()));
    TPE_TRY(up(o_akv, akv.data(), sizeof(double) * akv.size()));
    TPE_TRY(up(o_doff, doff.data(), sizeof(int32_t) * (nn + 1)));
    TPE_TRY(up(o_dsrc, dsrc.data(), sizeof(int32_t) * dsrc.size()));
    TPE_TRY(up(o_psi, h_psi, sizeof(double) * E * nr));
    const Node* dn = reinterpret_cast<const Node*>(base + o_nodes);
    const int32_t* dperm = reinterpret_cast<const int32_t*>(base + o_perm);
    const double* dmass = reinterpret_cast<const double*>(base + o_mass);
    const double* dpsi = reinterpret_cast<const double*>(base + o_psi);
    double* dmom = reinterpret_cast<double*>(base + o_mom);
    double* dloc = reinterpret_cast<double*>(base + o_loc);
    double* dphi = reinterpret_cast<double*>(base + o_phi);
    {
        KernelScope ks(ctx, TPE_KGROUP_PAIR_WEIGHTS, 3);
        bct_moment_kernel<<<(nn + 127) / 128, 128, 0, st>>>(dn, nn, dperm, dmass, dpsi, nr, dmom);
        TPE_CUDA_TRY(cudaGetLastError());
        bct_local_kernel<<<(nn + 127) / 128, 128, 0, st>>>(
            nn, reinterpret_cast<const int32_t*>(base + o_aoff), reinterpret_cast<const int32_t*>(base + o_asrc),
            reinterpret_cast<const double*>(base + o_akv), dmom, nr, dloc);
        TPE_CUDA_TRY(cudaGetLastError());
        bct_apply_kernel<<<(E + 127) / 128, 128, 0, st>>>(
            kind, d_xyz, ctx->d_edges.as<int2>(), E, dn, dperm, reinterpret_cast<const int32_t*>(base + o_leaf),
            dmass, dloc, reinterpret_cast<const int32_t*>(base + o_doff),
            reinterpret_cast<const int32_t*>(base + o_dsrc), dpsi, nr, eps, dphi);
        TPE_CUDA_TRY(cudaGetLastError());
    }
    TPE_CUDA_TRY(cudaMemcpyAsync(h_phi, dphi, sizeof(double) * E * nr, cudaMemcpyDeviceToHost, st));
    TPE_CUDA_TRY(cudaStreamSynchronize(st));
    if (stats) {
        stats[0] = L.admissible + L.direct_blocks;  // leaves of the block tree
        stats[1] = L.admissible;
        stats[2] = L.direct_blocks;
        stats[3] = L.direct_pairs;
    }
    return TPE_OK;
}

}  // namespace tpe

// The edge tree alone, on the host (no device, no context): for checking the
// builder against the stage-2 oracle's build_edge_bvh node by node.
extern "C" int32_t tpe_edge_tree(const double* xyz, int32_t V, const int32_t* edges, int32_t E,
                                 double epsilon, int32_t leaf_size, int32_t max_nodes,
                                 double* node_f, int32_t* node_i, int32_t* perm,
                                 int32_t* n_nodes) {
    try {
        if (!xyz || !edges || !node_f || !node_i || !perm || !n_nodes || V < 0 || E < 1 ||
            leaf_size < 1)
            return TPE_ERR_BAD_ARG;
        for (int64_t q = 0; q < 2 * (int64_t)E; q++)
            if (edges[q] < 0 || edges[q] >= V) return TPE_ERR_BAD_ARG;
        tpe::Tree tr;
        tpe::build_tree(edges, E, xyz, epsilon, leaf_size, tr);
        *n_nodes = (int32_t)tr.nodes.size();
        if ((int64_t)tr.nodes.size() > max_nodes) return TPE_ERR_TOO_LARGE;
        for (size_t i = 0; i < tr.nodes.size(); i++) {
            const tpe::Node& nd = tr.nodes[i];
            const double f[9] = {nd.cx, nd.cy, nd.cz, nd.tx, nd.ty, nd.tz, nd.mass, nd.rx, nd.rT};
            for (int q = 0; q < 9; q++) node_f[9 * i + q] = f[q];
            node_i[4 * i] = nd.begin;
            node_i[4 * i + 1] = nd.count;
            node_i[4 * i + 2] = nd.left;
            node_i[4 * i + 3] = nd.right;
        }
        for (int32_t k = 0; k < E; k++) perm[k] = tr.perm[k];
        return TPE_OK;
    } catch (const std::bad_alloc&) {
        return TPE_ERR_OUT_OF_MEMORY;
    } catch (...) {
        return TPE_ERR_INTERNAL;
    }
}
