// Host-side checks of the FP64 rho1 work lists that the plan builds (no GPU
// needed): chunking into ranges of consecutive batches, point tiles covering
// every batch exactly once, and the three work orders.  Built and run by
// tests/test_work_lists.py against libfrpa.so; prints "ok" or the first failure.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "frpa_internal.cuh"

using frpa::Rho1WorkItem;

static int fail_count = 0;
#define CHECK(cond, ...)                      \
  do {                                        \
    if (!(cond)) {                            \
      if (fail_count++ == 0) {                \
        std::printf("FAIL line %d: ", __LINE__); \
        std::printf(__VA_ARGS__);             \
        std::printf("\n");                    \
      }                                       \
    }                                         \
  } while (0)

static double cost(const Rho1WorkItem &w) { return (double)w.nc * w.nc * w.pn; }

int main() {
  std::mt19937 rng(7);
  for (int trial = 0; trial < 24; ++trial) {
    const int n_batches = trial < 4 ? trial + 1 : 50 + (int)(rng() % 400);
    std::vector<int> ib;
    std::vector<Rho1WorkItem> batches;
    for (int b = 0; b < n_batches; ++b) {
      if (rng() % 7 == 0) continue;  // a batch without compute functions: not in the plan's list
      const int nc = 1 + (int)(rng() % 600), np = (int)(rng() % 300);
      const int off = (int)ib.size();
      for (int i = 0; i < nc; ++i) ib.push_back(1 + (int)(rng() % 5000));
      batches.push_back(Rho1WorkItem{b, nc, np, 0, np, off, 0, frpa::rho1_locality_key(ib.data() + off, nc), 0});
    }
    double total = 0.0, biggest = 0.0;
    for (const Rho1WorkItem &b : batches) {
      total += (double)b.nc * b.nc * b.np;
      biggest = std::max(biggest, (double)b.nc * b.nc * b.np);
    }
    for (int tp : {64, 128})
      for (int order = 0; order <= 2; ++order) {
        std::vector<Rho1WorkItem> items;
        std::vector<int> ci, cb;
        frpa::rho1_fp64_build_items(batches, tp, order, n_batches, &items, &ci, &cb);
        CHECK((int)ci.size() == frpa::FP64_CHUNKS + 1 && (int)cb.size() == frpa::FP64_CHUNKS + 1,
              "chunk vectors of size %zu / %zu", ci.size(), cb.size());
        if (fail_count) break;
        CHECK(ci[0] == 0 && ci.back() == (int)items.size() && cb[0] == 0 && cb.back() == n_batches,
              "chunk ends %d..%d of %zu items, %d..%d of %d batches", ci[0], ci.back(), items.size(), cb[0],
              cb.back(), n_batches);
        // every point of every batch once, tiles of <= tp points, widths a multiple of 8 but the last
        std::vector<int> covered(n_batches, 0);
        for (int c = 0; c < frpa::FP64_CHUNKS; ++c) {
          CHECK(ci[c] <= ci[c + 1] && cb[c] <= cb[c + 1], "chunk %d bounds not increasing", c);
          double part = 0.0;
          for (int i = ci[c]; i < ci[c + 1]; ++i) {
            const Rho1WorkItem &w = items[i];
            CHECK(w.batch >= cb[c] && w.batch < cb[c + 1], "item of batch %d in chunk %d [%d, %d)", w.batch, c,
                  cb[c], cb[c + 1]);
            CHECK(w.pn >= 1 && w.pn <= tp && w.p0 + w.pn <= w.np, "tile %d+%d of %d points (tp %d)", w.p0, w.pn,
                  w.np, tp);
            CHECK(w.p0 % 8 == 0, "tile start %d not a multiple of 8", w.p0);
            CHECK(w.p0 == covered[w.batch], "batch %d: tile at %d after %d points", w.batch, w.p0,
                  covered[w.batch]);
            covered[w.batch] += w.pn;
            part += cost(w);
            if (i > ci[c]) {
              const Rho1WorkItem &v = items[i - 1];
              if (order == 0) CHECK(cost(v) >= cost(w), "order 0 not largest first");
              if (order == 1) CHECK(v.batch <= w.batch, "order 1 not in batch order");
              if (order == 2)
                CHECK((unsigned)v.key < (unsigned)w.key || (v.key == w.key && cost(v) >= cost(w)),
                      "order 2 not by key, largest first within a key");
            }
          }
          (void)part;
        }
        for (const Rho1WorkItem &b : batches)
          CHECK(covered[b.batch] == b.np, "batch %d: %d of %d points covered", b.batch, covered[b.batch], b.np);
        // the chunk boundaries split the cost at 6 / 50 / 94 %, up to one batch
        const double split[4] = {0.0, 0.06, 0.50, 0.94};
        for (int c = 1; c < frpa::FP64_CHUNKS; ++c) {
          double before = 0.0;
          for (const Rho1WorkItem &b : batches)
            if (b.batch < cb[c]) before += (double)b.nc * b.nc * b.np;
          CHECK(before >= split[c] * total - 1e-9 * total - biggest || cb[c] == n_batches,
                "chunk %d starts at %.3f of the cost", c, before / total);
          CHECK(before <= split[c] * total + biggest + 1e-9 * total, "chunk %d starts at %.3f of the cost", c,
                before / total);
        }
      }
  }
  // the locality key: the same list gives the same key, a superset never a larger one
  {
    std::vector<int> a = {3, 10, 11, 12, 400, 401}, b = {3, 10, 11, 12, 400, 401, 999};
    CHECK(frpa::rho1_locality_key(a.data(), (int)a.size()) == frpa::rho1_locality_key(a.data(), (int)a.size()),
          "key not deterministic");
    CHECK((unsigned)frpa::rho1_locality_key(b.data(), (int)b.size()) <=
              (unsigned)frpa::rho1_locality_key(a.data(), (int)a.size()),
          "key of a superset larger");
  }
  if (fail_count) return 1;
  std::printf("ok\n");
  return 0;
}
