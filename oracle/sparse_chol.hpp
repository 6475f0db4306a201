// Simplicial sparse Cholesky (LL^T) with a geometric nested-dissection ordering.
//
// TEST ORACLE ONLY.  It stands in for Eigen::SimplicialLLT<SparseMatrix<float>>, which the
// reference's CPU path calls every step (Cloth.cu:686-688).  Eigen is a third-party
// header library that is not present here (CMakeLists.txt:35 finds it on the system,
// with no pinned version).  Eigen's simplicial factorisation is the up-looking row-by-row
// algorithm over the elimination tree (Davis, "Direct Methods for Sparse Linear
// Systems", 2006, ch. 4); this file restates that published algorithm.  The fill-reducing
// ordering differs (Eigen defaults to AMD; this uses coordinate bisection nested
// dissection), which changes FP32 rounding but not the algorithm class or its cost order.
#ifndef CLOTHSTEP_SPARSE_CHOL_HPP
#define CLOTHSTEP_SPARSE_CHOL_HPP

#include <algorithm>
#include <cmath>
#include <vector>

namespace orc {

// Nested dissection on a graph with node coordinates (dim 2 or 3).  Returns order[new] = old.
inline std::vector<int> nestedDissection(int n, const int* rowPtr, const int* col, const double* xyz, int dim,
                                         int leaf = 48) {
    std::vector<int> order;
    order.reserve(n);
    std::vector<int> mark(n, 0);
    int stamp = 0;
    std::vector<int> ids(n);
    for (int i = 0; i < n; i++) ids[i] = i;
    // explicit stack to avoid deep recursion on large meshes
    struct Job { std::vector<int> ids; bool emit; };
    std::vector<Job> stack;
    stack.push_back({ids, false});
    while (!stack.empty()) {
        Job job = std::move(stack.back());
        stack.pop_back();
        if (job.emit || (int)job.ids.size() <= leaf) {
            order.insert(order.end(), job.ids.begin(), job.ids.end());
            continue;
        }
        std::vector<int>& s = job.ids;
        double lo[3] = {1e300, 1e300, 1e300}, hi[3] = {-1e300, -1e300, -1e300};
        for (int i : s)
            for (int d = 0; d < dim; d++) {
                lo[d] = std::min(lo[d], xyz[dim * i + d]);
                hi[d] = std::max(hi[d], xyz[dim * i + d]);
            }
        int ax = 0;
        for (int d = 1; d < dim; d++)
            if (hi[d] - lo[d] > hi[ax] - lo[ax]) ax = d;
        size_t mid = s.size() / 2;
        std::nth_element(s.begin(), s.begin() + mid, s.end(), [&](int a, int b) {
            double ca = xyz[dim * a + ax], cb = xyz[dim * b + ax];
            return ca < cb || (ca == cb && a < b);
        });
        std::vector<int> left(s.begin(), s.begin() + mid), right(s.begin() + mid, s.end());
        ++stamp;
        for (int i : right) mark[i] = stamp;
        std::vector<int> sep, left2;
        for (int i : left) {
            bool touches = false;
            for (int p = rowPtr[i]; p < rowPtr[i + 1]; p++)
                if (mark[col[p]] == stamp) { touches = true; break; }
            (touches ? sep : left2).push_back(i);
        }
        // emitted in reverse push order: left2, right, sep
        stack.push_back({sep, true});
        stack.push_back({right, false});
        stack.push_back({left2, false});
    }
    return order;
}

template <class T>
struct SparseCholesky {
    int n = 0;
    std::vector<int> perm, iperm;       // perm[new] = old
    std::vector<int> Cp, Ci;            // permuted upper triangle, by columns
    std::vector<int> srcIdx;            // index into the caller's CSR value array per Ci entry
    std::vector<int> parent, Lp, Li;
    std::vector<T> Lx;
    std::vector<int> work, stackBuf, cnext;
    std::vector<T> xbuf;

    // Symbolic analysis of a symmetric matrix given as full CSR (both triangles).
    void analyze(int nIn, const int* rp, const int* ci, const std::vector<int>& order) {
        n = nIn;
        perm = order;
        iperm.assign(n, 0);
        for (int k = 0; k < n; k++) iperm[perm[k]] = k;
        // upper triangle of C = P A P^T by columns: column k holds rows i <= k
        std::vector<int> cnt(n + 1, 0);
        for (int k = 0; k < n; k++) {
            int r = perm[k];
            for (int p = rp[r]; p < rp[r + 1]; p++)
                if (iperm[ci[p]] <= k) cnt[k + 1]++;
        }
        Cp.assign(n + 1, 0);
        for (int k = 0; k < n; k++) Cp[k + 1] = Cp[k] + cnt[k + 1];
        Ci.resize(Cp[n]);
        srcIdx.resize(Cp[n]);
        for (int k = 0; k < n; k++) {
            int r = perm[k], q = Cp[k];
            for (int p = rp[r]; p < rp[r + 1]; p++) {
                int i = iperm[ci[p]];
                if (i <= k) { Ci[q] = i; srcIdx[q] = p; q++; }
            }
        }
        // elimination tree (Davis 2006, sec. 4.1)
        parent.assign(n, -1);
        std::vector<int> anc(n, -1);
        for (int k = 0; k < n; k++) {
            for (int p = Cp[k]; p < Cp[k + 1]; p++) {
                int i = Ci[p];
                while (i != -1 && i < k) {
                    int nx = anc[i];
                    anc[i] = k;
                    if (nx == -1) parent[i] = k;
                    i = nx;
                }
            }
        }
        // column counts by row subtrees
        work.assign(n, -1);
        stackBuf.assign(n, 0);
        std::vector<int> colCount(n, 1);
        for (int k = 0; k < n; k++) {
            int top = ereach(k);
            for (int t = top; t < n; t++) colCount[stackBuf[t]]++;
        }
        Lp.assign(n + 1, 0);
        for (int k = 0; k < n; k++) Lp[k + 1] = Lp[k] + colCount[k];
        Li.resize(Lp[n]);
        Lx.resize(Lp[n]);
        xbuf.assign(n, T(0));
        cnext.resize(n);
    }

    // Pattern of row k of L, topologically ordered in stackBuf[top..n-1] (Davis 2006, sec. 4.2).
    int ereach(int k) {
        int top = n;
        work[k] = k;
        for (int p = Cp[k]; p < Cp[k + 1]; p++) {
            int i = Ci[p];
            if (i > k) continue;
            int len = 0;
            int* s = stackBuf.data();
            // walk up the etree until a marked node; record the path
            std::vector<int>& path = pathBuf;
            path.clear();
            while (work[i] != k) {
                path.push_back(i);
                work[i] = k;
                i = parent[i];
            }
            len = (int)path.size();
            while (len > 0) s[--top] = path[--len];
        }
        return top;
    }
    std::vector<int> pathBuf;

    // Numeric factorisation; returns false if the matrix is not positive definite.
    bool factor(const T* vals) {
        std::fill(work.begin(), work.end(), -1);
        for (int k = 0; k < n; k++) cnext[k] = Lp[k];
        for (int k = 0; k < n; k++) {
            int top = ereach(k);
            xbuf[k] = T(0);
            for (int p = Cp[k]; p < Cp[k + 1]; p++) xbuf[Ci[p]] = vals[srcIdx[p]];
            T d = xbuf[k];
            xbuf[k] = T(0);
            for (; top < n; top++) {
                int i = stackBuf[top];
                T lki = xbuf[i] / Lx[Lp[i]];
                xbuf[i] = T(0);
                for (int p = Lp[i] + 1; p < cnext[i]; p++) xbuf[Li[p]] -= Lx[p] * lki;
                d -= lki * lki;
                int p = cnext[i]++;
                Li[p] = k;
                Lx[p] = lki;
            }
            if (!(d > T(0))) return false;
            int p = cnext[k]++;
            Li[p] = k;
            Lx[p] = std::sqrt(d);
        }
        return true;
    }

    void solve(const T* b, T* x) const {
        std::vector<T> y(n);
        for (int k = 0; k < n; k++) y[k] = b[perm[k]];
        for (int j = 0; j < n; j++) {
            y[j] /= Lx[Lp[j]];
            for (int p = Lp[j] + 1; p < Lp[j + 1]; p++) y[Li[p]] -= Lx[p] * y[j];
        }
        for (int j = n - 1; j >= 0; j--) {
            for (int p = Lp[j] + 1; p < Lp[j + 1]; p++) y[j] -= Lx[p] * y[Li[p]];
            y[j] /= Lx[Lp[j]];
        }
        for (int k = 0; k < n; k++) x[perm[k]] = y[k];
    }

    long long nnzL() const { return Lp.empty() ? 0 : Lp[n]; }
};

}  // namespace orc

#endif
