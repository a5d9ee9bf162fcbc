// Host construction of the static front plan of the sparse LU (sparse.cuh).
#include <algorithm>
#include <iterator>
#include <numeric>

#include "sparse.cuh"

namespace alg {
namespace sp {

int build_front_plan(const Pattern& p, const Supernodal& S, int small_rows, int lanes, FrontPlan* out) {
  FrontPlan& F = *out;
  F = FrontPlan();
  const idx n = p.n, ns = S.n_supernodes(), nnz = p.nnz();
  F.n = n;
  F.nnz = nnz;
  F.ns = ns;
  F.col_perm.assign(S.col_perm.begin(), S.col_perm.end());
  F.fronts.assign(ns, FrontDesc{});
  if (n == 0) return SP_OK;
  const std::vector<idx>& ptr = S.supernode_ptr;
  std::vector<int32_t> owner(n);
  for (idx s = 0; s < ns; ++s)
    for (idx c = ptr[s]; c < ptr[s + 1]; ++c) owner[c] = (int32_t)s;

  // rows of A in positions: each row's columns (new positions) and the CSC
  // index of each entry
  std::vector<int64_t> rp(n + 1, 0);
  for (idx q = 0; q < nnz; ++q) rp[p.row_idx[q] + 1] += 1;
  for (idx r = 0; r < n; ++r) rp[r + 1] += rp[r];
  std::vector<int32_t> rpos((size_t)nnz);
  std::vector<int64_t> rq((size_t)nnz);
  {
    std::vector<int64_t> fill(rp.begin(), rp.end() - 1);
    for (idx c = 0; c < n; ++c)
      for (size_t q = p.col_ptr[c]; q < p.col_ptr[c + 1]; ++q) {
        const int64_t t = fill[p.row_idx[q]]++;
        rpos[t] = (int32_t)S.col_perm_inv[c];
        rq[t] = (int64_t)q;
      }
  }
  // the front each row enters: the owner of its first column
  std::vector<int32_t> leaf(n, -1);
  for (idx r = 0; r < n; ++r) {
    if (rp[r + 1] == rp[r]) {
      F.structurally_singular = true;  // an empty row
      continue;
    }
    int32_t lo = rpos[rp[r]];
    for (int64_t t = rp[r]; t < rp[r + 1]; ++t) lo = std::min(lo, rpos[t]);
    leaf[r] = owner[lo];
  }
  std::vector<int32_t> newptr(ns + 1, 0);
  for (idx r = 0; r < n; ++r)
    if (leaf[r] >= 0) newptr[leaf[r] + 1] += 1;
  for (idx s = 0; s < ns; ++s) newptr[s + 1] += newptr[s];
  F.new_rows.assign(newptr[ns], 0);
  {
    std::vector<int32_t> fill(newptr.begin(), newptr.end() - 1);
    for (idx r = 0; r < n; ++r)
      if (leaf[r] >= 0) F.new_rows[fill[leaf[r]]++] = (int32_t)r;  // increasing r within a front
  }
  // children in increasing order
  std::vector<int32_t> kptr(ns + 1, 0);
  for (idx s = 0; s < ns; ++s)
    if (S.super_etree[s] >= 0) kptr[S.super_etree[s] + 1] += 1;
  for (idx s = 0; s < ns; ++s) kptr[s + 1] += kptr[s];
  F.child_idx.assign(kptr[ns], 0);
  F.child_slot.assign(kptr[ns], 0);
  {
    std::vector<int32_t> fill(kptr.begin(), kptr.end() - 1);
    for (idx s = 0; s < ns; ++s)
      if (S.super_etree[s] >= 0) F.child_idx[fill[S.super_etree[s]]++] = (int32_t)s;
  }

  // fronts in postorder: slots, Struct(s), column maps
  std::vector<int32_t> mark(n, -1);
  std::vector<int32_t> loc_of(n, -1);             // position -> local column in the current front
  std::vector<int32_t> rloc((size_t)nnz, -1);     // local column of each row-form entry in its front
  std::vector<int32_t> sbeg(ns + 1, 0);
  std::vector<int32_t> cand, merged, extra;
  F.cb_colmap.clear();
  for (idx s = 0; s < ns; ++s) {
    FrontDesc& d = F.fronts[s];
    const int32_t b = (int32_t)ptr[s], e = (int32_t)ptr[s + 1];
    d.begin = b;
    d.size = e - b;
    d.child_begin = kptr[s];
    d.child_end = kptr[s + 1];
    d.new_begin = newptr[s];
    d.new_end = newptr[s + 1];
    // Struct(s): sorted union of the children's Struct (each sorted) and of
    // the entering rows' columns, restricted to columns after s
    int32_t slot = 0;
    cand.clear();
    for (int32_t k = d.child_begin; k < d.child_end; ++k) {
      const int32_t c = F.child_idx[k];
      const FrontDesc& dc = F.fronts[c];
      F.child_slot[k] = slot;
      slot += dc.rows - dc.size;
      const int32_t* lo = std::lower_bound(F.struct_cols.data() + sbeg[c], F.struct_cols.data() + sbeg[c + 1], e);
      const int32_t* hi = F.struct_cols.data() + sbeg[c + 1];
      if (cand.empty()) {
        cand.assign(lo, hi);
      } else {
        merged.clear();
        std::set_union(cand.begin(), cand.end(), lo, hi, std::back_inserter(merged));
        cand.swap(merged);
      }
    }
    extra.clear();
    for (int32_t k = d.new_begin; k < d.new_end; ++k) {
      const int32_t r = F.new_rows[k];
      for (int64_t t = rp[r]; t < rp[r + 1]; ++t) {
        const int32_t q = rpos[t];
        if (q >= e && mark[q] != s) {
          mark[q] = (int32_t)s;
          extra.push_back(q);
        }
      }
    }
    if (!extra.empty()) {
      std::sort(extra.begin(), extra.end());
      merged.clear();
      std::set_union(cand.begin(), cand.end(), extra.begin(), extra.end(), std::back_inserter(merged));
      cand.swap(merged);
    }
    d.rows = slot + (d.new_end - d.new_begin);
    if (d.rows < d.size) F.structurally_singular = true;
    sbeg[s] = (int32_t)F.struct_cols.size();
    d.struct_begin = sbeg[s];
    F.struct_cols.insert(F.struct_cols.end(), cand.begin(), cand.end());
    sbeg[s + 1] = (int32_t)F.struct_cols.size();
    d.ncb = (int32_t)cand.size();
    // the children's contribution columns in this front's local numbering
    for (int32_t j = b; j < e; ++j) loc_of[j] = j - b;
    for (int32_t t = 0; t < d.ncb; ++t) loc_of[cand[t]] = d.size + t;
    F.cb_colmap.resize(F.struct_cols.size());
    for (int32_t k = d.child_begin; k < d.child_end; ++k) {
      const int32_t c = F.child_idx[k];
      for (int32_t t = sbeg[c]; t < sbeg[c + 1]; ++t) F.cb_colmap[t] = loc_of[F.struct_cols[t]];
    }
    // local columns of the A entries of the rows entering here
    for (int32_t k = d.new_begin; k < d.new_end; ++k) {
      const int32_t r = F.new_rows[k];
      for (int64_t t = rp[r]; t < rp[r + 1]; ++t) rloc[t] = loc_of[rpos[t]];
    }
  }

  // A values of the entering rows: slot and local column in their front
  {
    std::vector<int32_t> cnt(ns + 1, 0);
    for (idx r = 0; r < n; ++r)
      if (leaf[r] >= 0) cnt[leaf[r] + 1] += (int32_t)(rp[r + 1] - rp[r]);
    for (idx s = 0; s < ns; ++s) cnt[s + 1] += cnt[s];
    F.anew_q.assign(cnt[ns], 0);
    F.anew_slot.assign(cnt[ns], 0);
    F.anew_col.assign(cnt[ns], 0);
    for (idx s = 0; s < ns; ++s) {
      FrontDesc& d = F.fronts[s];
      d.anew_begin = cnt[s];
      d.anew_end = cnt[s + 1];
      int32_t w = cnt[s];
      const int32_t slot0 = d.rows - (d.new_end - d.new_begin);
      for (int32_t k = d.new_begin; k < d.new_end; ++k) {
        const int32_t r = F.new_rows[k];
        for (int64_t t = rp[r]; t < rp[r + 1]; ++t) {
          F.anew_q[w] = rq[t];
          F.anew_slot[w] = slot0 + (k - d.new_begin);
          F.anew_col[w] = rloc[t];
          ++w;
        }
      }
    }
  }

  // small fronts: few rows, small block, every child small
  std::vector<int32_t> height(ns, 0);
  for (idx s = 0; s < ns; ++s) {
    FrontDesc& d = F.fronts[s];
    bool small = d.rows <= small_rows && (int64_t)d.rows * (d.size + d.ncb) <= (1 << 21);
    int32_t h = 0;
    for (int32_t k = d.child_begin; k < d.child_end; ++k) {
      const int32_t c = F.child_idx[k];
      small = small && F.fronts[c].small;
      h = std::max(h, height[c] + 1);
    }
    d.small = small ? 1 : 0;
    height[s] = h;
  }
  // offsets
  int64_t lo = 0, uo = 0, ro = 0, bo = 0;
  for (idx s = 0; s < ns; ++s) {
    FrontDesc& d = F.fronts[s];
    d.l_off = lo;
    lo += (int64_t)d.rows * d.size;
    d.u_off = uo;
    uo += (int64_t)d.size * d.ncb;
    d.rowid_off = ro;
    ro += d.rows;
    if (d.small) {
      d.block_off = bo;
      bo += (int64_t)d.rows * (d.size + d.ncb);
      d.cb_off = d.block_off + d.size + (int64_t)d.size * d.rows;
      d.cb_ld = d.rows;
    } else {
      d.block_off = -1;
    }
    const double m = d.rows, k = d.size, c = d.ncb;
    F.flops += 2.0 * k * k * m - 2.0 / 3.0 * k * k * k + k * k * c + 2.0 * (m - k) * c * k;
  }
  F.l_total = lo;
  F.u_total = uo;
  F.rowid_total = ro;
  F.block_total = bo;
  // large fronts: postorder, split into lanes (independent subtrees factored
  // concurrently, one stream each) and the fronts above them; contribution
  // blocks on one stack per lane and one for the top, in disjoint regions
  {
    std::vector<int32_t> big_parent(ns, -1);
    std::vector<double> cost(ns, 0.0), sub(ns, 0.0);
    for (idx s = 0; s < ns; ++s) {
      FrontDesc& d = F.fronts[s];
      if (d.small) continue;
      F.big_order.push_back((int32_t)s);
      for (int32_t k = d.child_begin; k < d.child_end; ++k)
        if (!F.fronts[F.child_idx[k]].small) big_parent[F.child_idx[k]] = (int32_t)s;
      // seconds: updates at ~15 TFLOP/s, contribution-block traffic at ~3 TB/s,
      // a launch chain and a column-serial panel
      const double m = d.rows, k = d.size, c = d.ncb;
      const double fl = 2.0 * k * k * m - 2.0 / 3.0 * k * k * k + k * k * c + 2.0 * (m - k) * c * k;
      cost[s] = fl / 15e12 + 24.0 * (m - k) * c / 3e12 + 50e-6 + 5e-6 * k;
    }
    for (int32_t s : F.big_order) {  // children precede parents
      sub[s] += cost[s];
      if (big_parent[s] >= 0) sub[big_parent[s]] += sub[s];
    }
    // split the heaviest subtree at its root (the root goes to the top) until
    // the lanes can be balanced
    std::vector<int32_t> tasks;
    std::vector<char> is_top(ns, 0);
    for (int32_t s : F.big_order)
      if (big_parent[s] < 0) tasks.push_back(s);
    const int K = std::max(1, std::min(lanes, 8));
    while (K > 1 && !tasks.empty() && tasks.size() < 64) {
      size_t hi = 0;
      double total = 0.0;
      for (size_t i = 0; i < tasks.size(); ++i) {
        total += sub[tasks[i]];
        if (sub[tasks[i]] > sub[tasks[hi]]) hi = i;
      }
      const int32_t r = tasks[hi];
      if ((int)tasks.size() >= K && sub[r] <= 1.1 * total / K) break;
      const FrontDesc& d = F.fronts[r];
      std::vector<int32_t> kids;
      for (int32_t k = d.child_begin; k < d.child_end; ++k)
        if (!F.fronts[F.child_idx[k]].small) kids.push_back(F.child_idx[k]);
      if (kids.empty()) break;
      is_top[r] = 1;
      tasks.erase(tasks.begin() + hi);
      tasks.insert(tasks.end(), kids.begin(), kids.end());
    }
    // longest-processing-time assignment of the subtrees to lanes
    std::sort(tasks.begin(), tasks.end(), [&](int32_t x, int32_t y) { return sub[x] > sub[y]; });
    std::vector<double> load(K, 0.0);
    std::vector<int32_t> lane_of(ns, -1);
    for (int32_t r : tasks) {
      const int k = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      load[k] += sub[r];
      lane_of[r] = k;
    }
    // every front of a task's subtree takes the task's lane (parents come
    // later in postorder, so walk the order backwards)
    for (auto it = F.big_order.rbegin(); it != F.big_order.rend(); ++it) {
      const int32_t s = *it;
      if (is_top[s] || lane_of[s] >= 0) continue;
      lane_of[s] = lane_of[big_parent[s]];
    }
    F.n_lanes = K;
    F.lane_ptr.assign(K + 1, 0);
    F.lane_front_buf.assign(K, 0);
    for (int32_t s : F.big_order)
      if (!is_top[s]) F.lane_ptr[lane_of[s] + 1] += 1;
    for (int k = 0; k < K; ++k) F.lane_ptr[k + 1] += F.lane_ptr[k];
    F.lane_fronts.assign(F.lane_ptr[K], 0);
    std::vector<int32_t> fill(F.lane_ptr.begin(), F.lane_ptr.end() - 1);
    for (int32_t s : F.big_order) {
      if (is_top[s])
        F.top_fronts.push_back(s);
      else
        F.lane_fronts[fill[lane_of[s]]++] = s;
    }
    // stacks: lane k's region, then the top's; a front pops the contribution
    // blocks of its large children on its own stack (the lanes' roots are
    // read in place by the top fronts)
    int64_t base = 0;
    auto run_stack = [&](const int32_t* list, int cnt, bool top, int64_t* fbuf) {
      std::vector<std::pair<int64_t, int64_t>> stack;  // (offset, length)
      int64_t at = base, peak = base;
      for (int i = 0; i < cnt; ++i) {
        FrontDesc& d = F.fronts[list[i]];
        *fbuf = std::max(*fbuf, (int64_t)d.rows * (d.size + d.ncb));
        int npop = 0;
        for (int32_t k = d.child_begin; k < d.child_end; ++k) {
          const int32_t c = F.child_idx[k];
          if (!F.fronts[c].small && (!top || is_top[c])) ++npop;
        }
        for (int q = 0; q < npop; ++q) {
          at = stack.back().first;
          stack.pop_back();
        }
        d.cb_off = at;
        d.cb_ld = std::max(1, d.rows - d.size);
        const int64_t len = (int64_t)(d.rows - d.size) * d.ncb;
        stack.push_back({at, len});
        at += len;
        peak = std::max(peak, at);
      }
      base = peak;
    };
    for (int k = 0; k < K; ++k)
      run_stack(F.lane_fronts.data() + F.lane_ptr[k], F.lane_ptr[k + 1] - F.lane_ptr[k], false,
                &F.lane_front_buf[k]);
    run_stack(F.top_fronts.data(), (int)F.top_fronts.size(), true, &F.lane_front_buf[0]);
    F.stack_total = base;
    F.front_buf = 0;
    for (int64_t fb : F.lane_front_buf) F.front_buf = std::max(F.front_buf, fb);
  }
  // levels: small fronts (batched kernel) and all fronts (solve)
  {
    int32_t hmax = 0;
    for (idx s = 0; s < ns; ++s) hmax = std::max(hmax, height[s]);
    std::vector<int32_t> cs(hmax + 2, 0), ca(hmax + 2, 0);
    for (idx s = 0; s < ns; ++s) {
      if (F.fronts[s].small) cs[height[s] + 1] += 1;
      ca[height[s] + 1] += 1;
    }
    for (int32_t h = 0; h <= hmax; ++h) {
      cs[h + 1] += cs[h];
      ca[h + 1] += ca[h];
    }
    F.small_level_ptr = cs;
    F.solve_level_ptr = ca;
    F.small_level_fronts.assign(cs[hmax + 1], 0);
    F.solve_level_fronts.assign(ca[hmax + 1], 0);
    std::vector<int32_t> fs(cs.begin(), cs.end() - 1), fa(ca.begin(), ca.end() - 1);
    for (idx s = 0; s < ns; ++s) {
      if (F.fronts[s].small) F.small_level_fronts[fs[height[s]]++] = (int32_t)s;
      F.solve_level_fronts[fa[height[s]]++] = (int32_t)s;
    }
    // drop trailing empty small levels
    while (F.small_level_ptr.size() > 1 &&
           F.small_level_ptr[F.small_level_ptr.size() - 1] == F.small_level_ptr[F.small_level_ptr.size() - 2])
      F.small_level_ptr.pop_back();
  }
  // A by rows (for the mixed form's FP64 residual): entries of each row in
  // column order, with their CSC index
  {
    F.csr_ptr.assign(n + 1, 0);
    for (idx q = 0; q < nnz; ++q) F.csr_ptr[p.row_idx[q] + 1] += 1;
    for (idx i = 0; i < n; ++i) F.csr_ptr[i + 1] += F.csr_ptr[i];
    F.csr_col.assign(nnz, 0);
    F.csr_map.assign(nnz, 0);
    std::vector<int64_t> next(F.csr_ptr.begin(), F.csr_ptr.end() - 1);
    for (idx j = 0; j < n; ++j)
      for (size_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) {
        const int64_t at = next[p.row_idx[q]]++;
        F.csr_col[at] = (int32_t)j;
        F.csr_map[at] = (int64_t)q;
      }
  }
  return SP_OK;
}


// Merges a front's last child (the one just before it in postorder, so the
// merged columns stay contiguous) into it when the merged front's flops stay
// within (1 + tol) of the two separate fronts', or, for two large fronts,
// when the extra flops cost less than the child's contribution-block traffic
// and launch chain (times traffic_scale; 0 turns that rule off): a merged step no longer copies the whole contribution
// block into the next front. The merged front of a child c and its parent s
// has size_c + size_s columns, rows_s + size_c rows and the parent's Struct
// (c's Struct outside s's columns is contained in s's); the parent's other
// children become the merged front's children (their rows are zero in c's
// columns, as they are sibling subtrees of c). Pivots do not depend on the
// partition.
// Break-even of merging a chain child into its parent: FP64 tensor-core
// flops per HBM byte of the dense updates (about 15 TFLOP/s against 3 TB/s
// of effective front traffic), and the flops one front's launch chain
// (panels, TRSM, assembly, about 50 us) is worth.
constexpr double kFlopsPerByte = 5.0;
constexpr double kFrontOverheadFlops = 7.5e8;

void amalgamate_chains(const FrontPlan& F, const Supernodal& S, double tol, double traffic_scale,
                       std::vector<idx>* ptr_out) {
  const idx ns = F.ns;
  auto flops = [](double m, double k, double c) {
    return 2.0 * k * k * m - 2.0 / 3.0 * k * k * k + k * k * c + 2.0 * (m - k) * c * k;
  };
  std::vector<double> gm(ns), gk(ns), gc(ns);
  std::vector<char> into_next(ns, 0);
  for (idx s = 0; s < ns; ++s) {
    const FrontDesc& d = F.fronts[s];
    gm[s] = d.rows;
    gk[s] = d.size;
    gc[s] = d.ncb;
    if (s > 0 && S.super_etree[s - 1] == s) {  // s - 1 is s's last child (postorder)
      const double m2 = d.rows + gk[s - 1], k2 = d.size + gk[s - 1], c2 = d.ncb;
      const double sep = flops(gm[s - 1], gk[s - 1], gc[s - 1]) + flops(d.rows, d.size, d.ncb);
      // a separate child front costs its contribution block's HBM traffic
      // (written after its update, read back by the parent's assembly, about
      // three passes) and a fixed launch chain; merged, those extra flops
      // run inside the parent's updates instead
      // (only between large fronts: a small front's columns stay in the
      // batched kernel, off the large fronts' column-serial panel chain)
      const double cb_bytes = 24.0 * (gm[s - 1] - gk[s - 1]) * gc[s - 1];
      const double saved = traffic_scale * (kFlopsPerByte * cb_bytes + kFrontOverheadFlops);
      const double merged = flops(m2, k2, c2);
      const bool both_large = !F.fronts[s - 1].small && !d.small;
      if (merged <= (1.0 + tol) * sep || (both_large && merged - sep <= saved)) {
        into_next[s - 1] = 1;
        gm[s] = m2;
        gk[s] = k2;
        gc[s] = c2;
      }
    }
  }
  ptr_out->assign(1, 0);
  for (idx s = 0; s < ns; ++s)
    if (!into_next[s]) ptr_out->push_back(S.supernode_ptr[s + 1]);
}

void repartition(const Supernodal& S, const std::vector<idx>& ptr, Supernodal* out) {
  *out = S;
  out->supernode_ptr = ptr;
  const idx ns = (idx)ptr.size() - 1;
  std::vector<idx> owner(S.n);
  for (idx s = 0; s < ns; ++s)
    for (idx c = ptr[s]; c < ptr[s + 1]; ++c) owner[c] = s;
  out->super_etree.assign(ns, -1);
  for (idx s = 0; s < ns; ++s) {
    const idx last = ptr[s + 1] - 1;
    if (S.etree[last] >= 0) out->super_etree[s] = owner[S.etree[last]];
  }
}

void split_at_etree_breaks(const Supernodal& S, Supernodal* out) {
  std::vector<idx> ptr(1, 0);
  for (idx s = 0; s < S.n_supernodes(); ++s) {
    for (idx j = S.supernode_ptr[s] + 1; j < S.supernode_ptr[s + 1]; ++j)
      if (S.etree[j - 1] != j) ptr.push_back(j);
    ptr.push_back(S.supernode_ptr[s + 1]);
  }
  repartition(S, ptr, out);
}

}  // namespace sp
}  // namespace alg
