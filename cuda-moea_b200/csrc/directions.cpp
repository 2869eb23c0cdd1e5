// Das-Dennis reference directions on the host.
//
// Reference: python/csrc/native/src/reference/nsga3_reference_generator.cu:28-221
// and rvea_reference_generator.cu:18-205.  The point order is the order in
// which std::prev_permutation enumerates the bar positions of a stars-and-bars
// mask, and the FP32 normalisation is the reference's (v / sqrtf(sum v^2) for
// the population-size form, v * (1 / sqrt(sum v^2)) for the partitions form),
// because association ties are broken by direction index.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "moea_b200.h"
#include "dirtree.h"

namespace moea {

int set_error(int code, const char* fmt, ...);

namespace {

long long combinations(int n, int k)
{
    if (k > n) return 0;
    if (k == 0 || k == n) return 1;
    k = std::min(k, n - k);
    long long r = 1;
    for (int i = 1; i <= k; ++i) {
        r *= (n - k + i);
        r /= i;
    }
    return r;
}

// One layer of h partitions in M objectives, objective-major into out
// starting at column col0 of a matrix with `stride` columns.
void layer(int h, int M, std::vector<float>& out, int stride, int col0)
{
    const int len = h + M - 1;
    std::vector<bool> bars(len, false);
    std::fill(bars.begin(), bars.begin() + (M - 1), true);
    std::vector<int> cut(M + 1);
    int point = 0;
    do {
        int c = 0;
        cut[c++] = -1;
        for (int i = 0; i < len; ++i)
            if (bars[i]) cut[c++] = i;
        cut[c] = len;
        for (int m = 0; m < M; ++m)
            out[(size_t)m * stride + col0 + point] = (cut[m + 1] - cut[m] - 1) / static_cast<float>(h);
        ++point;
    } while (std::prev_permutation(bars.begin(), bars.end()));
}

}  // namespace

// mode 0: NSGA-III from the population size, 1: NSGA-III by partitions,
// 2: RVEA from the population size.  Returns count or -1.
int das_dennis(int mode, int n, int M, std::vector<float>& out)
{
    if (M <= 0) return -1;
    if (mode == 1) {
        if (n <= 0) return -1;
        const long long c = combinations(n + M - 1, M - 1);
        if (c <= 0 || c > (1 << 26)) return -1;
        const int count = (int)c;
        out.assign((size_t)M * count, 0.0f);
        layer(n, M, out, count, 0);
        for (int p = 0; p < count; ++p) {
            float norm2 = 0.0f;
            for (int m = 0; m < M; ++m) {
                const float v = out[(size_t)m * count + p];
                norm2 += v * v;
            }
            const float inverse = 1.0f / std::sqrt(norm2);
            for (int m = 0; m < M; ++m) out[(size_t)m * count + p] = out[(size_t)m * count + p] * inverse;
        }
        return count;
    }
    if (n < 1) return -1;
    int h1 = 0;
    while (combinations(h1 + M - 1, M - 1) <= n) ++h1;
    --h1;
    if (h1 < 1) return -1;
    const int n1 = (int)combinations(h1 + M - 1, M - 1);
    int n2 = 0, h2 = 0;
    if (h1 < M) {
        h2 = 1;
        while (combinations(h1 + M - 1, M - 1) + combinations(h2 + M - 1, M - 1) <= n) ++h2;
        --h2;
        if (h2 > 0) n2 = (int)combinations(h2 + M - 1, M - 1);
    }
    const int count = n1 + n2;
    out.assign((size_t)M * count, 0.0f);
    layer(h1, M, out, count, 0);
    if (n2 > 0) {
        layer(h2, M, out, count, n1);
        const float centroid = 1.0f / M;
        for (int p = 0; p < n2; ++p)
            for (int m = 0; m < M; ++m) {
                float& v = out[(size_t)m * count + n1 + p];
                v = 0.5f * (v + centroid);
            }
    }
    if (mode == 2)
        for (float& v : out) v = std::max(v, 1e-6f);
    for (int p = 0; p < count; ++p) {
        float sum_sq = 0.0f;
        for (int m = 0; m < M; ++m) {
            const float v = out[(size_t)m * count + p];
            sum_sq += v * v;
        }
        const float norm = sqrtf(sum_sq);
        for (int m = 0; m < M; ++m) out[(size_t)m * count + p] = out[(size_t)m * count + p] / norm;
    }
    return count;
}

// User-defined directions, optionally normalised to unit length
// (nat/src/reference/reference_directions.cu:186-235).
int normalize_user_directions(std::vector<float>& v, int M, int count)
{
    for (int k = 0; k < count; ++k) {
        float norm2 = 0.0f;
        for (int m = 0; m < M; ++m) {
            const float value = v[(size_t)m * count + k];
            norm2 += value * value;
        }
        if (norm2 <= 0.0f) return set_error(MOEA_ERR_INVALID_ARGUMENT, "Reference directions must be non-zero");
        const float inverse = 1.0f / std::sqrt(norm2);
        for (int m = 0; m < M; ++m) v[(size_t)m * count + k] *= inverse;
    }
    return MOEA_OK;
}

// Cone tree over the directions for the pruned association search.
//
// Directions are reordered so that every node covers a contiguous range of
// the new order.  A node with more than kTreeLeaf directions gets up to 32
// children by five levels of median splits along the coordinate of largest
// spread; a node with at most kTreeLeaf directions is a leaf.  Nodes are
// numbered breadth first, so the children of a node are contiguous.  Each
// node stores the unit mean of its members' unit vectors and a cone around it
// that contains every member (cos and sin of the half angle, rounded
// outwards).  delta = max | |r|^2 - 1 | over the directions.
namespace {

constexpr int kTreeLeaf = 32;

int median_split(const float* refs, int M, int H, std::vector<int>& order, int lo, int hi)
{
    int axis = 0;
    float best = -1.0f;
    for (int m = 0; m < M; ++m) {
        float mn = INFINITY, mx = -INFINITY;
        for (int i = lo; i < hi; ++i) {
            const float v = refs[(size_t)m * H + order[i]];
            mn = std::min(mn, v);
            mx = std::max(mx, v);
        }
        if (mx - mn > best) { best = mx - mn; axis = m; }
    }
    const int mid = lo + (hi - lo) / 2;
    std::nth_element(order.begin() + lo, order.begin() + mid, order.begin() + hi, [&](int a, int b) {
        const float va = refs[(size_t)axis * H + a], vb = refs[(size_t)axis * H + b];
        return va < vb || (va == vb && a < b);
    });
    return mid;
}

void expand(const float* refs, int M, int H, std::vector<int>& order, int lo, int hi, int levels,
            std::vector<std::pair<int, int>>& out)
{
    if (hi - lo <= kTreeLeaf || levels == 0) {
        out.push_back({lo, hi});
        return;
    }
    const int mid = median_split(refs, M, H, order, lo, hi);
    expand(refs, M, H, order, lo, mid, levels - 1, out);
    expand(refs, M, H, order, mid, hi, levels - 1, out);
}

}  // namespace

int build_direction_tree(const float* refs, int M, int H, DirectionTreeHost& t)
{
    t = DirectionTreeHost{};
    t.M = M;
    t.H = H;
    t.order.resize(H);
    for (int j = 0; j < H; ++j) t.order[j] = j;
    double delta = 0.0;
    std::vector<double> unit((size_t)M * H);
    for (int j = 0; j < H; ++j) {
        double rr = 0.0;
        for (int m = 0; m < M; ++m) rr += (double)refs[(size_t)m * H + j] * refs[(size_t)m * H + j];
        if (!std::isfinite(rr)) delta = INFINITY;
        else delta = std::max(delta, std::fabs(rr - 1.0));
        const double inv = rr > 0.0 ? 1.0 / std::sqrt(rr) : 0.0;
        for (int m = 0; m < M; ++m) unit[(size_t)m * H + j] = refs[(size_t)m * H + j] * inv;
    }
    t.delta = (float)std::min(delta, 1e30);
    std::vector<std::pair<int, int>> ranges{{0, H}};
    std::vector<int> depth{0};
    for (size_t k = 0; k < ranges.size(); ++k) {
        const int lo = ranges[k].first, hi = ranges[k].second;
        t.max_depth = std::max(t.max_depth, depth[k] + 1);
        if (hi - lo <= kTreeLeaf) {
            t.link.push_back(lo);
            t.link.push_back(-(hi - lo));
            continue;
        }
        std::vector<std::pair<int, int>> kids;
        expand(refs, M, H, t.order, lo, hi, 5, kids);
        t.link.push_back((int)ranges.size());
        t.link.push_back((int)kids.size());
        for (auto& c : kids) {
            ranges.push_back(c);
            depth.push_back(depth[k] + 1);
        }
    }
    const int nodes = (int)ranges.size();
    t.nodes = nodes;
    t.center.assign((size_t)M * nodes, 0.0f);
    t.cos_r.assign(nodes, -1.0f);
    t.sin_r.assign(nodes, 1.0f);
    std::vector<double> c(M);
    for (int k = 0; k < nodes; ++k) {
        const int lo = ranges[k].first, hi = ranges[k].second;
        std::fill(c.begin(), c.end(), 0.0);
        for (int i = lo; i < hi; ++i)
            for (int m = 0; m < M; ++m) c[m] += unit[(size_t)m * H + t.order[i]];
        double norm = 0.0;
        for (int m = 0; m < M; ++m) norm += c[m] * c[m];
        norm = std::sqrt(norm);
        if (!(norm > 1e-12)) continue;  // no cone: the node is never pruned
        for (int m = 0; m < M; ++m) c[m] /= norm;
        double cmin = 1.0;
        for (int i = lo; i < hi; ++i) {
            double dot = 0.0;
            for (int m = 0; m < M; ++m) dot += c[m] * unit[(size_t)m * H + t.order[i]];
            cmin = std::min(cmin, dot);
        }
        cmin = std::max(-1.0, cmin - 1e-6);
        const double smax = std::min(1.0, std::sqrt(std::max(0.0, 1.0 - cmin * cmin)) + 1e-6);
        for (int m = 0; m < M; ++m) t.center[(size_t)m * nodes + k] = (float)c[m];
        t.cos_r[k] = std::nextafter((float)cmin, -2.0f);
        t.sin_r[k] = std::min(1.0f, std::nextafter((float)smax, 2.0f));
    }
    t.dirs.resize((size_t)M * H);
    for (int m = 0; m < M; ++m)
        for (int i = 0; i < H; ++i) t.dirs[(size_t)m * H + i] = refs[(size_t)m * H + t.order[i]];
    return MOEA_OK;
}

}  // namespace moea

extern "C" moea_status moea_reference_directions(int mode, int n, int M, float* h_out,
                                                 size_t capacity, int* h_count)
{
    if (!h_count || mode < 0 || mode > 2)
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "reference_directions: bad arguments");
    std::vector<float> out;
    const int count = moea::das_dennis(mode, n, M, out);
    if (count < 0)
        return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "reference_directions: invalid request (mode=%d n=%d M=%d)",
                               mode, n, M);
    *h_count = count;
    if (h_out) {
        if (capacity < out.size())
            return moea::set_error(MOEA_ERR_INVALID_ARGUMENT, "reference_directions: capacity %zu < %zu",
                                   capacity, out.size());
        std::memcpy(h_out, out.data(), out.size() * sizeof(float));
    }
    return MOEA_OK;
}
