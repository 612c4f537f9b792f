// Locality order of an operator's rows for the persistent recursions.
//
// A recursion step reads, for every row, the rows of its neighbours in T_n.  On a 3D
// lattice numbered x + L(y + Lz) the z neighbours lie L^2 rows away, so at 8e6 sites and
// 64 vector columns a neighbour row is evicted from L2 before the sweep comes back to it
// and T_n is read from HBM about three times per step.  Visiting the rows in an order in
// which graph neighbours are close in time keeps them in L2; the data stay where they are
// (each row of a block is R contiguous values), only the traversal changes, so the results
// are the same up to the order of the per-CTA dot-product sums.
//
// The order is found from the sparsity pattern alone, by recursive graph bisection: a
// part of the row graph is ordered breadth-first from a pseudo-peripheral row (the last row
// reached by a breadth-first search from its first row) and split into the first and the
// second half of that order; the halves are split again until they have at most `part`
// rows.  A leaf keeps the breadth-first order of its parent, so the rows of a leaf are
// compact in the graph and those of consecutive leaves mostly border each other.  The parts
// of one level are independent and run on host threads.
#include "internal.cuh"

#include <atomic>
#include <thread>

namespace linqt {
namespace {

struct Range {
  int b, e;
};

// Breadth-first order of the rows in order[b, e) (label == b), from `root`, restarting from
// the first unvisited row of the range when a component is exhausted; writes the order to q
// and returns the last row reached.
int bfs_part(const int *rp, const int *ci, const int *label, int *mark, int stamp, const int *order, int b, int e,
             int root, std::vector<int> &q) {
  q.clear();
  int scan = b;
  for (;;) {
    mark[root] = stamp;
    size_t head = q.size();
    q.push_back(root);
    while (head < q.size()) {
      const int v = q[head++];
      for (int k = rp[v]; k < rp[v + 1]; ++k) {
        const int u = ci[k];
        if (label[u] == b && mark[u] != stamp) {
          mark[u] = stamp;
          q.push_back(u);
        }
      }
    }
    if ((int)q.size() == e - b) break;
    while (mark[order[scan]] == stamp) ++scan;  // another component of the part
    root = order[scan];
  }
  return q.back();
}

}  // namespace

std::vector<int> locality_order(int n, const int *rp, const int *ci, int part) {
  std::vector<int> order(n), label(n, 0), next(n, 0), mark(n, -1);
  for (int i = 0; i < n; ++i) order[i] = i;
  if (n <= part) return order;
  std::vector<Range> work{{0, n}};
  const int nth = (int)std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
  for (int level = 0; !work.empty(); ++level) {
    std::vector<std::vector<Range>> out(nth);
    std::atomic<size_t> cursor{0};
    auto worker = [&](int t) {
      std::vector<int> q;
      for (size_t i; (i = cursor.fetch_add(1)) < work.size();) {
        const Range r = work[i];
        // two searches: the first finds a pseudo-peripheral row, the second orders from it
        const int far = bfs_part(rp, ci, label.data(), mark.data(), 2 * level, order.data(), r.b, r.e,
                                 order[r.b], q);
        bfs_part(rp, ci, label.data(), mark.data(), 2 * level + 1, order.data(), r.b, r.e, far, q);
        std::copy(q.begin(), q.end(), order.begin() + r.b);
        const int mid = r.b + (r.e - r.b) / 2;
        for (int k = mid; k < r.e; ++k) next[order[k]] = mid;
        for (const Range c : {Range{r.b, mid}, Range{mid, r.e}})
          if (c.e - c.b > part) out[t].push_back(c);
      }
    };
    // parts of a level only read `label` and write `order`, `mark` and `next` at their own rows
    if (work.size() == 1 || nth == 1) {
      worker(0);
    } else {
      std::vector<std::thread> pool;
      for (int t = 0; t < nth; ++t) pool.emplace_back(worker, t);
      for (auto &th : pool) th.join();
    }
    label = next;
    work.clear();
    for (auto &v : out) work.insert(work.end(), v.begin(), v.end());
  }
  return order;
}

}  // namespace linqt
