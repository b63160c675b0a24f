// Host construction of the Hall basis and of the Lie <-> tensor maps.
//
// The Hall set is built by the same greedy rule as RoughPy
// (roughpy/compute/_src/lie_basis.c:201-337; libalgebra_lite
// basis/hall_set.cpp:81-106): letters are keys 1..d; for each degree, for
// each left degree l <= degree/2, keys i of degree l and j > i of degree
// degree-l form the key (i, j) whenever left_parent(j) <= i.
//
// l2t expands a key to its tensor polynomial, [a, b] -> ab - ba.
// t2l maps a word a_1..a_k to r(a_1..a_k)/k where r is right-normed
// bracketing r(a u) = [a, r(u)] (lie_basis.c:1066-1200, maps.h:175-210);
// [a, r(u)] is rewritten into the Hall basis by the classical Jacobi
// rewriting [x, (y1, y2)] = [[x, y1], y2] + [y1, [x, y2]] for non-Hall pairs.
// Because the Hall elements form a basis, the expansion (and thus the map)
// is unique, so any correct rewriting reproduces the reference matrix.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <unordered_map>
#include <vector>

#include "common.cuh"

namespace rpyb {
namespace {

using LieVec = std::map<int64_t, int64_t>;   // key -> integer coefficient

struct HallSet {
    int width = 0, depth = 0;
    std::vector<int64_t> left, right;     // parents per key (key 0 = null)
    std::vector<int64_t> degree_begin;    // size depth + 2
    std::vector<int> deg;                 // degree per key
    std::map<std::pair<int64_t, int64_t>, int64_t> reverse;

    int64_t size() const { return (int64_t)left.size() - 1; }
};

std::unique_ptr<HallSet> build_hall_set(int width, int depth)
{
    auto h = std::make_unique<HallSet>();
    h->width = width;
    h->depth = depth;
    h->degree_begin.assign(depth + 2, 0);
    h->left.push_back(0);
    h->right.push_back(0);
    h->deg.push_back(0);
    if (depth > 0) {
        h->degree_begin[1] = 1;
        for (int a = 1; a <= width; ++a) {
            h->left.push_back(0);
            h->right.push_back(a);
            h->deg.push_back(1);
        }
        h->degree_begin[2] = (int64_t)h->left.size();
    }
    for (int degree = 2; degree <= depth; ++degree) {
        for (int ld = 1; 2 * ld <= degree; ++ld) {
            const int rd = degree - ld;
            const int64_t i_lo = h->degree_begin[ld], i_hi = h->degree_begin[ld + 1];
            const int64_t j_lo = h->degree_begin[rd], j_hi = h->degree_begin[rd + 1];
            for (int64_t i = i_lo; i < i_hi; ++i) {
                for (int64_t j = std::max(i + 1, j_lo); j < j_hi; ++j) {
                    if (h->left[j] <= i) {
                        h->reverse[{i, j}] = (int64_t)h->left.size();
                        h->left.push_back(i);
                        h->right.push_back(j);
                        h->deg.push_back(degree);
                    }
                }
            }
            h->degree_begin[degree + 1] = (int64_t)h->left.size();
        }
    }
    for (int64_t a = 1; a <= width && depth > 0; ++a) h->reverse[{0, a}] = a;
    return h;
}

class Rewriter {
public:
    explicit Rewriter(const HallSet& h) : h_(h) {}

    // [x, y] for Hall keys, expanded in the Hall basis (truncated at depth).
    const LieVec& prod(int64_t x, int64_t y)
    {
        const auto keyp = std::make_pair(x, y);
        auto it = memo_.find(keyp);
        if (it != memo_.end()) return it->second;
        LieVec res;
        if (x != y && h_.deg[x] + h_.deg[y] <= h_.depth) {
            if (x > y) {
                const LieVec& r = prod(y, x);
                for (auto& [k, c] : r) res[k] = -c;
            } else if (h_.deg[y] == 1 || h_.left[y] <= x) {
                res[h_.reverse.at({x, y})] = 1;
            } else {
                const int64_t y1 = h_.left[y], y2 = h_.right[y];
                // [[x, y1], y2]
                const LieVec a = prod(x, y1);
                for (auto& [k, c] : a) {
                    const LieVec& t = prod(k, y2);
                    for (auto& [k2, c2] : t) res[k2] += c * c2;
                }
                // [y1, [x, y2]]
                const LieVec b = prod(x, y2);
                for (auto& [k, c] : b) {
                    const LieVec& t = prod(y1, k);
                    for (auto& [k2, c2] : t) res[k2] += c * c2;
                }
                for (auto it2 = res.begin(); it2 != res.end();) {
                    if (it2->second == 0) it2 = res.erase(it2);
                    else ++it2;
                }
            }
        }
        return memo_.emplace(keyp, std::move(res)).first->second;
    }

private:
    const HallSet& h_;
    std::map<std::pair<int64_t, int64_t>, LieVec> memo_;
};

struct LieMaps {
    std::unique_ptr<HallSet> hall;
    // CSR, float64
    std::vector<int64_t> l2t_ptr, l2t_idx;
    std::vector<double> l2t_val;
    std::vector<int64_t> t2l_ptr, t2l_idx;
    std::vector<double> t2l_val;
};

std::unique_ptr<LieMaps> build_maps(int width, int depth)
{
    auto m = std::make_unique<LieMaps>();
    m->hall = build_hall_set(width, depth);
    const HallSet& h = *m->hall;
    Geometry g;
    make_geometry(width, depth, g);
    const int64_t T = g.size();
    const int64_t L = h.size();

    // ---- l2t: tensor expansion of each key (sparse word -> coefficient)
    std::vector<std::map<int64_t, int64_t>> expand(L + 1);   // word index within level
    for (int64_t k = 1; k <= L; ++k) {
        if (h.deg[k] == 1) {
            expand[k][h.right[k] - 1] = 1;
            continue;
        }
        const int64_t a = h.left[k], b = h.right[k];
        const int da = h.deg[a], dbb = h.deg[b];
        for (auto& [wa, ca] : expand[a])
            for (auto& [wb, cb] : expand[b]) {
                expand[k][wa * g.pw[dbb] + wb] += ca * cb;
                expand[k][wb * g.pw[da] + wa] -= ca * cb;
            }
        for (auto it = expand[k].begin(); it != expand[k].end();) {
            if (it->second == 0) it = expand[k].erase(it);
            else ++it;
        }
    }
    {
        // rows = tensor index, cols = lie index (key - 1)
        std::vector<std::vector<std::pair<int64_t, double>>> rows(T);
        for (int64_t k = 1; k <= L; ++k)
            for (auto& [w, c] : expand[k]) rows[g.db[h.deg[k]] + w].push_back({k - 1, (double)c});
        m->l2t_ptr.assign(T + 1, 0);
        for (int64_t r = 0; r < T; ++r) {
            std::sort(rows[r].begin(), rows[r].end());
            m->l2t_ptr[r + 1] = m->l2t_ptr[r] + (int64_t)rows[r].size();
            for (auto& [c, v] : rows[r]) {
                m->l2t_idx.push_back(c);
                m->l2t_val.push_back(v);
            }
        }
    }

    // ---- t2l: r(word)/degree, built level by level from suffixes
    Rewriter rw(h);
    std::vector<LieVec> rprev, rcur;   // r(word) for words of the previous / current level
    std::vector<std::vector<std::pair<int64_t, double>>> cols_per_lie(L);  // lie row -> entries
    for (int k = 1; k <= depth; ++k) {
        rcur.assign(g.pw[k], LieVec());
        const double inv = 1.0 / (double)k;
        for (int64_t w = 0; w < g.pw[k]; ++w) {
            LieVec& r = rcur[w];
            if (k == 1) {
                r[w + 1] = 1;
            } else {
                const int64_t first = 1 + w / g.pw[k - 1];   // letter key
                const int64_t suffix = w % g.pw[k - 1];
                for (auto& [key, c] : rprev[suffix]) {
                    const LieVec& p = rw.prod(first, key);
                    for (auto& [k2, c2] : p) r[k2] += c * c2;
                }
                for (auto it = r.begin(); it != r.end();) {
                    if (it->second == 0) it = r.erase(it);
                    else ++it;
                }
            }
            for (auto& [key, c] : r)
                cols_per_lie[key - 1].push_back({g.db[k] + w, (double)c * inv});
        }
        rprev.swap(rcur);
    }
    m->t2l_ptr.assign(L + 1, 0);
    for (int64_t i = 0; i < L; ++i) {
        std::sort(cols_per_lie[i].begin(), cols_per_lie[i].end());
        m->t2l_ptr[i + 1] = m->t2l_ptr[i] + (int64_t)cols_per_lie[i].size();
        for (auto& [c, v] : cols_per_lie[i]) {
            m->t2l_idx.push_back(c);
            m->t2l_val.push_back(v);
        }
    }
    return m;
}

std::mutex g_maps_mu;
std::map<std::pair<int, int>, std::unique_ptr<LieMaps>> g_maps;

const LieMaps* get_maps(int width, int depth)
{
    std::lock_guard<std::mutex> lk(g_maps_mu);
    auto key = std::make_pair(width, depth);
    auto it = g_maps.find(key);
    if (it != g_maps.end()) return it->second.get();
    auto m = build_maps(width, depth);
    return g_maps.emplace(key, std::move(m)).first->second.get();
}

int check_lie_args(int32_t width, int32_t depth)
{
    Geometry g;
    int rc = make_geometry(width, depth, g);
    if (rc) return rc;
    if (depth < 1) return fail(RPYB_E_INVALID, "Lie basis needs depth >= 1");
    if (g.size() > (int64_t(1) << 24))
        return fail(RPYB_E_UNSUPPORTED, "Lie maps limited to tensors of at most 2^24 scalars");
    return RPYB_OK;
}

}  // namespace
}  // namespace rpyb

using namespace rpyb;

extern "C" {

RPYB_API int64_t rpyb_lie_basis_size(int32_t width, int32_t depth)
{
    if (check_lie_args(width, depth)) return -1;
    return get_maps(width, depth)->hall->size();
}

RPYB_API int rpyb_lie_basis_data(int32_t width, int32_t depth, int64_t* data,
                                 int64_t* degree_begin)
{
    int rc = check_lie_args(width, depth);
    if (rc) return rc;
    const HallSet& h = *get_maps(width, depth)->hall;
    if (data) {
        for (int64_t k = 0; k <= h.size(); ++k) {
            data[2 * k] = h.left[k];
            data[2 * k + 1] = h.right[k];
        }
    }
    if (degree_begin) std::memcpy(degree_begin, h.degree_begin.data(), sizeof(int64_t) * (depth + 2));
    return RPYB_OK;
}

RPYB_API int64_t rpyb_lie_map_csr(int32_t width, int32_t depth, int which, int64_t* indptr,
                                  int64_t* indices, double* values)
{
    int rc = check_lie_args(width, depth);
    if (rc) return rc;
    if (which != 0 && which != 1) return fail(RPYB_E_INVALID, "which must be 0 (l2t) or 1 (t2l)");
    const LieMaps* m = get_maps(width, depth);
    const auto& ptr = which == 0 ? m->l2t_ptr : m->t2l_ptr;
    const auto& idx = which == 0 ? m->l2t_idx : m->t2l_idx;
    const auto& val = which == 0 ? m->l2t_val : m->t2l_val;
    if (indices == nullptr && values == nullptr && indptr == nullptr) return (int64_t)idx.size();
    if (indptr) std::memcpy(indptr, ptr.data(), sizeof(int64_t) * ptr.size());
    if (indices) std::memcpy(indices, idx.data(), sizeof(int64_t) * idx.size());
    if (values) std::memcpy(values, val.data(), sizeof(double) * val.size());
    return (int64_t)idx.size();
}

}  // extern "C"
