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
    int32_t begin, count;  // the node's edges: perm[begin .. begin + count)
    int32_t left, right;   // children, -1 for a leaf
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

struct Builder {
    const std::vector<double>& C;  // E x 3 midpoints
    const std::vector<double>& T;  // E x 3 unit tangents
    const std::vector<double>& m;  // E masses (ell_eps)
    int32_t leaf;
    std::vector<int32_t> perm;
    std::vector<Node> nodes;
    std::vector<double> tmp;

    int32_t rec(int32_t begin, int32_t count) {
        const int32_t* idx = perm.data() + begin;
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
        nodes.push_back(Node{c[0], c[1], c[2], msum, rx, rT, begin, count, -1, -1});
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
            std::stable_sort(perm.begin() + begin, perm.begin() + begin + count,
                             [&](int32_t a, int32_t b) { return X[3 * (size_t)a + dd] < X[3 * (size_t)b + dd]; });
            const int32_t mid = count / 2;
            const int32_t l = rec(begin, mid);
            const int32_t r = rec(begin + mid, count - mid);
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
    // edge geometry as edge_geometry computes it (tpe_stage2_oracle.py:72-82)
    std::vector<double> C((size_t)3 * E), T((size_t)3 * E), m((size_t)E);
    for (int32_t I = 0; I < E; I++) {
        const int32_t a = ctx->h_edges[2 * (size_t)I], b = ctx->h_edges[2 * (size_t)I + 1];
        double e[3];
        for (int d = 0; d < 3; d++) {
            e[d] = h_xyz[3 * (size_t)b + d] - h_xyz[3 * (size_t)a + d];
            C[3 * (size_t)I + d] = 0.5 * (h_xyz[3 * (size_t)a + d] + h_xyz[3 * (size_t)b + d]);
        }
        const double ell = norm3(e[0], e[1], e[2]);
        for (int d = 0; d < 3; d++) T[3 * (size_t)I + d] = ell >= kTangentTol ? e[d] / ell : 0.0;
        m[I] = ell + eps;
    }
    Builder B{C, T, m, leaf, {}, {}, {}};
    B.perm.resize((size_t)E);
    std::iota(B.perm.begin(), B.perm.end(), 0);
    B.nodes.reserve(2 * (size_t)E / std::max(1, leaf) + 2);
    B.rec(0, E);
    std::vector<int32_t> where((size_t)E);
    for (int32_t k = 0; k < E; k++) where[B.perm[k]] = k;
    const size_t nn = B.nodes.size();
    const size_t bytes_nodes = sizeof(Node) * nn, bytes_idx = sizeof(int32_t) * (size_t)E;
    const size_t off_perm = (bytes_nodes + 255) / 256 * 256;
    const size_t off_where = off_perm + (bytes_idx + 255) / 256 * 256;
    const size_t off_val = off_where + (bytes_idx + 255) / 256 * 256;
    const size_t off_cnt = off_val + (sizeof(double) * (size_t)E + 255) / 256 * 256;
    const size_t off_tot = off_cnt + (sizeof(long long) * 3 * (size_t)E + 255) / 256 * 256;
    TPE_TRY(ensure(ctx, ctx->bh_buf, off_tot + 256));
    uint8_t* base = ctx->bh_buf.as<uint8_t>();
    const cudaStream_t st = ctx->stream;
    TPE_CUDA_TRY(cudaMemcpyAsync(base, B.nodes.data(), bytes_nodes, cudaMemcpyHostToDevice, st));
    TPE_CUDA_TRY(cudaMemcpyAsync(base + off_perm, B.perm.data(), bytes_idx, cudaMemcpyHostToDevice, st));
    TPE_CUDA_TRY(cudaMemcpyAsync(base + off_where, where.data(), bytes_idx, cudaMemcpyHostToDevice, st));
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

}  // namespace tpe
