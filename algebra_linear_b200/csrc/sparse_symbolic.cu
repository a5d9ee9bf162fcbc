// Host-side symbolic analysis of the sparse LU (see sparse_symbolic.cuh).
//
// COLAMD follows the algorithm of src/sparse/faer/colamd.rs (faer's
// transcription of SuiteSparse COLAMD): the same column/row records with
// signed sentinels, the same dense row/column thresholds, bucket lists by
// approximate score, pivot-row construction, set-difference marks with
// aggressive absorption, hashing and super-column detection, garbage
// collection of the index array, and the postorder through the column
// elimination tree at the end. Every tie is broken exactly as there, so the
// permutation is identical.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>

#include "sparse_symbolic.cuh"

namespace alg {
namespace sp {

int validate_csc(size_t nrows, size_t ncols, const size_t* col_ptr, size_t col_ptr_len, const size_t* row_idx,
                 size_t row_idx_len) {
  if (col_ptr_len != ncols + 1) return SP_BAD_SHAPE;
  if (col_ptr[0] != 0) return SP_INVALID_STRUCTURE;
  if (col_ptr[ncols] != row_idx_len) return SP_BAD_SHAPE;
  for (size_t w = 1; w <= ncols; ++w)
    if (col_ptr[w] < col_ptr[w - 1]) return SP_INVALID_STRUCTURE;
  for (size_t k = 0; k < row_idx_len; ++k)
    if (row_idx[k] >= nrows) return SP_INVALID_STRUCTURE;
  for (size_t j = 0; j < ncols; ++j)
    for (size_t k = col_ptr[j] + 1; k < col_ptr[j + 1]; ++k) {
      if (row_idx[k - 1] == row_idx[k]) return SP_DUPLICATE_ENTRY;
      if (row_idx[k - 1] > row_idx[k]) return SP_UNSORTED_ROWS;
    }
  return SP_OK;
}

uint64_t fingerprint(const Pattern& p) {
  uint64_t h = 0xcbf29ce484222325ull;
  auto mix = [&](uint64_t x) {
    for (int b = 0; b < 8; ++b) {
      h ^= (x >> (8 * b)) & 0xffu;
      h *= 0x00000100000001b3ull;
    }
  };
  for (idx j = 0; j <= p.n; ++j) mix((uint64_t)p.col_ptr[j]);
  for (idx k = 0; k < p.nnz(); ++k) mix((uint64_t)p.row_idx[k]);
  return h;
}

// --------------------------------------------------------------------------
// Elimination tree and postorder
// --------------------------------------------------------------------------
void col_etree(const Pattern& p, const idx* perm, std::vector<idx>* etree_out) {
  const idx n = p.n;
  std::vector<idx>& parent = *etree_out;
  parent.assign(n, -1);
  std::vector<idx> anc(n, -1), last_col(n, -1);  // last_col[row]: latest column seen in that row
  for (idx j = 0; j < n; ++j) {
    const idx src = perm ? perm[j] : j;
    for (size_t q = p.col_ptr[src]; q < p.col_ptr[src + 1]; ++q) {
      const idx row = (idx)p.row_idx[q];
      idx i = last_col[row];
      while (i >= 0 && i != j) {
        const idx up = anc[i];
        anc[i] = j;  // path compression toward j
        if (up < 0) {
          parent[i] = j;
          break;
        }
        i = up;
      }
      last_col[row] = j;
    }
  }
}

void postorder(const std::vector<idx>& parent, std::vector<idx>* post_out) {
  const idx n = (idx)parent.size();
  std::vector<idx>& post = *post_out;
  post.assign(n, 0);
  if (n == 0) return;
  // children lists in increasing order (built from the highest index down)
  std::vector<idx> child(n, -1), sibling(n, -1), stack(n);
  for (idx j = n - 1; j >= 0; --j)
    if (parent[j] >= 0) {
      sibling[j] = child[parent[j]];
      child[parent[j]] = j;
    }
  idx out = 0;
  for (idx root = 0; root < n; ++root) {
    if (parent[root] >= 0) continue;
    idx top = 0;
    stack[top++] = root;
    while (top > 0) {
      const idx v = stack[top - 1];
      const idx c = child[v];
      if (c >= 0) {
        child[v] = sibling[c];  // consume the child, descend into it
        stack[top++] = c;
      } else {
        post[out++] = v;
        --top;
      }
    }
  }
}

// --------------------------------------------------------------------------
// COLAMD
// --------------------------------------------------------------------------
namespace {

struct ColRec {
  idx start, length;
  idx thick;  // thickness (>0), negated while marked; parent super-column once absorbed
  idx score;  // approximate score; order once eliminated
  idx prev;   // score-list predecessor; hash bucket while in a hash list
  idx next;   // score-list successor; hash-list successor
  bool dead() const { return start < 0; }
  bool dead_principal() const { return start == -1; }
};

struct RowRec {
  idx start, length;
  idx degree;  // external degree; also a cursor while transposing
  idx mark;    // <0: dead; set-difference mark otherwise; first column while compacting
  bool dead() const { return mark < 0; }
};

idx reset_marks(idx tag, idx limit, std::vector<RowRec>& rows) {
  if (tag == 0 || tag >= limit) {
    for (auto& r : rows)
      if (!r.dead()) r.mark = 0;
    return 1;
  }
  return tag;
}

// Compacts the column lists (dropping dead rows) and the row lists (dropping
// dead columns) to the front of the index array; returns the first free slot.
idx compact(std::vector<RowRec>& row, std::vector<ColRec>& col, std::vector<idx>& a, idx pfree, idx m, idx n) {
  idx dst = 0;
  for (idx c = 0; c < n; ++c) {
    if (col[c].dead()) continue;
    const idx s0 = col[c].start, len = col[c].length;
    col[c].start = dst;
    for (idx q = s0; q < s0 + len; ++q) {
      const idx r = a[q];
      if (!row[r].dead()) a[dst++] = r;
    }
    col[c].length = dst - col[c].start;
  }
  // tag the first entry of every live row with its (complemented) index
  for (idx r = 0; r < m; ++r) {
    if (row[r].dead() || row[r].length == 0) {
      row[r].mark = -1;
    } else {
      const idx q = row[r].start;
      row[r].mark = a[q];
      a[q] = ~r;
    }
  }
  idx src = dst;
  while (src < pfree) {
    if (a[src++] < 0) {
      --src;
      const idx r = ~a[src];
      a[src] = row[r].mark;
      row[r].start = dst;
      const idx len = row[r].length;
      for (idx t = 0; t < len; ++t) {
        const idx c = a[src++];
        if (!col[c].dead()) a[dst++] = c;
      }
      row[r].length = dst - row[r].start;
    }
  }
  return dst;
}

// Merges columns of the pivot row whose row lists are identical (same hash
// bucket, same length, same score) into super-columns.
void merge_identical_columns(std::vector<ColRec>& col, const std::vector<idx>& a, std::vector<idx>& head, idx rs,
                             idx rlen) {
  for (idx q = rs; q < rs + rlen; ++q) {
    const idx c0 = a[q];
    if (col[c0].dead()) continue;
    const idx bucket = col[c0].prev;
    const idx hcol = head[bucket];
    idx sc = hcol > -1 ? col[hcol].prev : -(hcol + 2);
    while (sc != -1) {
      const idx len = col[sc].length;
      idx before = sc;
      idx c = col[sc].next;
      while (c != -1) {
        bool same = col[c].length == len && col[c].score == col[sc].score;
        if (same) {
          const idx p1 = col[sc].start, p2 = col[c].start;
          for (idx t = 0; t < len; ++t)
            if (a[p1 + t] != a[p2 + t]) {
              same = false;
              break;
            }
        }
        if (!same) {
          before = c;
          c = col[c].next;
          continue;
        }
        col[sc].thick += col[c].thick;
        col[c].thick = sc;
        col[c].start = -2;  // dead, non-principal
        col[c].score = -1;
        col[before].next = col[c].next;
        c = col[c].next;
      }
      sc = col[sc].next;
    }
    if (hcol > -1)
      col[hcol].prev = -1;
    else
      head[bucket] = -1;
  }
}

}  // namespace

int colamd_order(const Pattern& pat, double dense_row, double dense_col, bool aggressive, std::vector<idx>* perm_out,
                 std::vector<idx>* perm_inv_out) {
  const idx n = pat.n, m = pat.n;
  perm_out->clear();
  perm_inv_out->clear();
  if (n == 0) return SP_OK;
  const idx nnz = pat.nnz();
  // index array of 2 nnz + nnz/5 + n entries
  const idx size = 2 * nnz + nnz / 5 + n;
  if (nnz < 0 || size < nnz) return SP_INDEX_OVERFLOW;
  std::vector<ColRec> col(n + 1);
  std::vector<RowRec> row(m + 1);
  std::vector<idx> head(n + 1, 0);
  std::vector<idx> a(size, 0);
  for (idx j = 0; j < n; ++j) {
    head[j + 1] = head[j] + (idx)(pat.col_ptr[j + 1] - pat.col_ptr[j]);
    for (idx t = 0; t < head[j + 1] - head[j]; ++t) a[head[j] + t] = (idx)pat.row_idx[pat.col_ptr[j] + t];
  }
  for (idx c = 0; c < n; ++c) col[c] = ColRec{head[c], head[c + 1] - head[c], 1, 0, -1, -1};
  col[n] = ColRec{-1, -1, -1, -1, -1, -1};
  for (idx r = 0; r < m; ++r) row[r] = RowRec{0, 0, -1, -1};
  row[m] = RowRec{-1, -1, -1, -1};

  // row lengths, then the row-form copy of the pattern after the column form
  for (idx c = 0; c < n; ++c)
    for (idx q = head[c]; q < head[c + 1]; ++q) {
      const idx r = a[q];
      row[r].length += 1;
      row[r].mark = c;
    }
  row[0].start = head[n];
  row[0].degree = row[0].start;
  row[0].mark = -1;
  for (idx r = 1; r < m; ++r) {
    row[r].start = row[r - 1].start + row[r - 1].length;
    row[r].degree = row[r].start;
    row[r].mark = -1;
  }
  for (idx c = 0; c < n; ++c)
    for (idx q = head[c]; q < head[c + 1]; ++q) {
      const idx r = a[q];
      a[row[r].degree++] = c;
    }
  for (idx r = 0; r < m; ++r) {
    row[r].mark = 0;
    row[r].degree = row[r].length;
  }

  const idx dense_row_count = dense_row < 0.0 ? n - 1 : std::max<idx>(16, (idx)(dense_row * (double)n));
  const idx dense_col_count =
      dense_col < 0.0 ? m - 1 : std::max<idx>(16, (idx)(dense_col * (double)std::min(m, n)));

  idx max_deg = 0;
  idx ncol2 = n;
  // empty columns go last (visited from the highest index)
  for (idx c = n - 1; c >= 0; --c)
    if (col[c].length == 0) {
      col[c].score = --ncol2;
      col[c].start = -1;
    }
  // dense columns next; each of their rows loses one degree
  for (idx c = n - 1; c >= 0; --c) {
    if (col[c].dead()) continue;
    if (col[c].length > dense_col_count) {
      col[c].score = --ncol2;
      for (idx q = col[c].start; q < col[c].start + col[c].length; ++q) row[a[q]].degree -= 1;
      col[c].start = -1;
    }
  }
  // dense and empty rows leave the graph
  for (idx r = 0; r < m; ++r) {
    const idx deg = row[r].degree;
    if (deg > dense_row_count || deg == 0)
      row[r].mark = -1;
    else
      max_deg = std::max(max_deg, deg);
  }
  // initial scores: sum over live rows of (degree - 1), capped at n
  for (idx c = n - 1; c >= 0; --c) {
    if (col[c].dead()) continue;
    idx score = 0, w = col[c].start;
    for (idx q = col[c].start; q < col[c].start + col[c].length; ++q) {
      const idx r = a[q];
      if (row[r].dead()) continue;
      a[w++] = r;
      score = std::min(score + row[r].degree - 1, n);
    }
    const idx len = w - col[c].start;
    if (len == 0) {
      col[c].score = --ncol2;
      col[c].start = -1;
    } else {
      col[c].length = len;
      col[c].score = score;
    }
  }
  // score buckets (doubly linked; head[score] is the first column)
  std::fill(head.begin(), head.end(), (idx)-1);
  for (idx c = n - 1; c >= 0; --c) {
    if (col[c].dead()) continue;
    const idx s = col[c].score;
    const idx nx = head[s];
    col[c].prev = -1;
    col[c].next = nx;
    if (nx != -1) col[nx].prev = c;
    head[s] = c;
  }

  const idx mark_limit = std::numeric_limits<idx>::max() - n;
  idx tag = reset_marks(0, mark_limit, row);
  idx min_score = 0;
  idx pfree = 2 * nnz;
  idx k = 0;
  while (k < ncol2) {
    while (head[min_score] == -1 && min_score < n) ++min_score;
    const idx pc = head[min_score];
    {
      const idx nx = col[pc].next;
      head[min_score] = nx;
      if (nx != -1) col[nx].prev = -1;
    }
    const idx pc_score = col[pc].score;
    col[pc].score = k;
    const idx pc_thick = col[pc].thick;
    k += pc_thick;
    const idx needed = std::min(pc_score, n - k);
    if (pfree + needed >= size) {
      pfree = compact(row, col, a, pfree, m, n);
      tag = reset_marks(0, mark_limit, row);
    }

    // the pivot row: union of the live columns of the pivot column's rows
    const idx prs = pfree;
    idx prdeg = 0;
    col[pc].thick = -pc_thick;
    for (idx q = col[pc].start; q < col[pc].start + col[pc].length; ++q) {
      const idx r = a[q];
      if (row[r].dead()) continue;
      for (idx t = row[r].start; t < row[r].start + row[r].length; ++t) {
        const idx c = a[t];
        const idx th = col[c].thick;
        if (th > 0 && !col[c].dead()) {
          col[c].thick = -th;
          a[pfree++] = c;
          prdeg += th;
        }
      }
    }
    col[pc].thick = pc_thick;
    max_deg = std::max(max_deg, prdeg);
    for (idx q = col[pc].start; q < col[pc].start + col[pc].length; ++q) row[a[q]].mark = -1;
    const idx prlen = pfree - prs;
    const idx prow = prlen > 0 ? a[col[pc].start] : -1;

    // unlink the pivot row's columns from their buckets; set-difference marks
    for (idx q = prs; q < prs + prlen; ++q) {
      const idx c = a[q];
      const idx th = -col[c].thick;
      col[c].thick = th;
      const idx s = col[c].score, pv = col[c].prev, nx = col[c].next;
      if (pv == -1)
        head[s] = nx;
      else
        col[pv].next = nx;
      if (nx != -1) col[nx].prev = pv;
      for (idx t = col[c].start; t < col[c].start + col[c].length; ++t) {
        const idx r = a[t];
        const idx mk = row[r].mark;
        if (row[r].dead()) continue;
        idx diff = mk - tag;
        if (diff < 0) diff = row[r].degree;
        diff -= th;
        if (diff == 0 && aggressive)
          row[r].mark = -1;
        else
          row[r].mark = diff + tag;
      }
    }

    // new scores of the pivot row's columns; hash them for super-columns
    for (idx q = prs; q < prs + prlen; ++q) {
      const idx c = a[q];
      idx hash = 0, score = 0, w = col[c].start;
      for (idx t = col[c].start; t < col[c].start + col[c].length; ++t) {
        const idx r = a[t];
        const idx mk = row[r].mark;
        if (row[r].dead()) continue;
        a[w++] = r;
        hash += r;
        score = std::min(score + (mk - tag), n);
      }
      col[c].length = w - col[c].start;
      if (col[c].length == 0) {
        col[c].start = -1;
        prdeg -= col[c].thick;
        col[c].score = k;
        k += col[c].thick;
      } else {
        col[c].score = score;
        hash %= n + 1;
        const idx hcol = head[hash];
        idx first;
        if (hcol > -1) {
          first = col[hcol].prev;
          col[hcol].prev = c;
        } else {
          first = -(hcol + 2);
          head[hash] = -(c + 2);
        }
        col[c].next = first;
        col[c].prev = hash;
      }
    }
    merge_identical_columns(col, a, head, prs, prlen);
    col[pc].start = -1;
    tag = reset_marks(tag + max_deg + 1, mark_limit, row);

    // the pivot row joins every surviving column; re-bucket by the new score
    idx w = prs;
    for (idx q = prs; q < prs + prlen; ++q) {
      const idx c = a[q];
      if (col[c].dead()) continue;
      a[w++] = c;
      a[col[c].start + col[c].length] = prow;
      col[c].length += 1;
      idx s = col[c].score + prdeg;
      const idx smax = n - k - col[c].thick;
      s -= col[c].thick;
      s = std::min(s, smax);
      col[c].score = s;
      const idx nx = head[s];
      col[c].next = nx;
      col[c].prev = -1;
      if (nx != -1) col[nx].prev = c;
      head[s] = c;
      min_score = std::min(min_score, s);
    }
    if (prdeg > 0) {
      row[prow].start = prs;
      row[prow].length = w - prs;
      row[prow].degree = prdeg;
      row[prow].mark = 0;
    }
  }

  // absorbed (non-principal) columns take consecutive orders after their
  // super-column's, then the order is read out
  for (idx i = 0; i < n; ++i) {
    if (!col[i].dead_principal() && col[i].score == -1) {
      idx parent = i;
      do {
        parent = col[parent].thick;
      } while (!col[parent].dead_principal());
      idx c = i, ord = col[parent].score;
      do {
        col[c].score = ord++;
        col[c].thick = parent;
        c = col[c].thick;
      } while (col[c].score == -1);
      col[parent].score = ord;
    }
  }
  std::vector<idx> perm(n), perm_inv(n);
  for (idx c = 0; c < n; ++c) perm[col[c].score] = c;
  for (idx c = 0; c < n; ++c) perm_inv[perm[c]] = c;

  // postorder through the column elimination tree of the ordered matrix
  std::vector<idx> et, post;
  col_etree(pat, perm.data(), &et);
  postorder(et, &post);
  for (idx i = 0; i < n; ++i) perm[post[i]] = i;                 // inverse postorder
  for (idx i = 0; i < n; ++i) perm_inv[i] = perm[perm_inv[i]];   // compose
  for (idx i = 0; i < n; ++i) perm[perm_inv[i]] = i;
  *perm_out = std::move(perm);
  *perm_inv_out = std::move(perm_inv);
  return SP_OK;
}

// --------------------------------------------------------------------------
// Column counts of chol(A^T A) and supernodes
// --------------------------------------------------------------------------
namespace {

// Row-form (transposed) pattern with sorted column indices.
void transpose(const Pattern& p, std::vector<size_t>* tp, std::vector<size_t>* ti) {
  const idx n = p.n;
  tp->assign(n + 1, 0);
  for (idx q = 0; q < p.nnz(); ++q) (*tp)[p.row_idx[q] + 1] += 1;
  for (idx r = 0; r < n; ++r) (*tp)[r + 1] += (*tp)[r];
  std::vector<size_t> fill(tp->begin(), tp->end() - 1);
  ti->assign(p.nnz(), 0);
  for (idx j = 0; j < n; ++j)
    for (size_t q = p.col_ptr[j]; q < p.col_ptr[j + 1]; ++q) (*ti)[fill[p.row_idx[q]]++] = (size_t)j;
}

// Skeleton-leaf test with path-compressed ancestors (the LCA step of the
// column-count algorithm): -2 if j is not a leaf of i's row subtree, -1 for
// the first leaf, else the least common ancestor with the previous leaf.
idx leaf_lca(idx i, idx j, const std::vector<idx>& first, std::vector<idx>& max_first, std::vector<idx>& prev_leaf,
             std::vector<idx>& anc) {
  if (i <= j || first[j] <= max_first[i]) return -2;
  max_first[i] = first[j];
  const idx jprev = prev_leaf[i];
  prev_leaf[i] = j;
  if (jprev < 0) return -1;
  idx q = jprev;
  while (q != anc[q]) q = anc[q];
  for (idx v = jprev; v != q;) {
    const idx up = anc[v];
    anc[v] = q;
    v = up;
  }
  return q;
}

std::vector<idx> counts_ata(idx n, const std::vector<size_t>& tp, const std::vector<size_t>& ti,
                            const std::vector<idx>& perm_inv, const std::vector<idx>& parent,
                            const std::vector<idx>& post) {
  std::vector<idx> delta(n, 0), first(n, -1), max_first(n, -1), prev_leaf(n, -1), anc(n), nxt(n, -1), head(n, -1),
      post_pos(n);
  for (idx i = 0; i < n; ++i) anc[i] = i;
  for (idx i = 0; i < n; ++i) post_pos[post[i]] = i;
  // rows of A bucketed by the earliest postorder position among their columns
  for (idx r = 0; r < n; ++r) {
    idx lo = std::numeric_limits<idx>::max();
    for (size_t q = tp[r]; q < tp[r + 1]; ++q) lo = std::min(lo, post_pos[perm_inv[ti[q]]]);
    if (lo != std::numeric_limits<idx>::max()) {
      nxt[r] = head[lo];
      head[lo] = r;
    }
  }
  for (idx k = 0; k < n; ++k) {
    idx v = post[k];
    delta[v] = first[v] < 0 ? 1 : 0;
    while (first[v] < 0) {
      first[v] = k;
      if (parent[v] < 0) break;
      v = parent[v];
    }
  }
  for (idx k = 0; k < n; ++k) {
    const idx v = post[k];
    if (parent[v] >= 0) delta[parent[v]] -= 1;
    idx r = head[k];
    head[k] = -1;
    for (; r >= 0; r = nxt[r])
      for (size_t q = tp[r]; q < tp[r + 1]; ++q) {
        const idx i = perm_inv[ti[q]];
        const idx lca = leaf_lca(i, v, first, max_first, prev_leaf, anc);
        if (lca != -2) {
          delta[v] += 1;
          if (lca >= 0) delta[lca] -= 1;
        }
      }
    if (parent[v] >= 0) anc[v] = parent[v];
  }
  for (idx v = 0; v < n; ++v)
    if (parent[v] >= 0) delta[parent[v]] += delta[v];
  return delta;
}

void tree_of_partition(const std::vector<idx>& ptr, const std::vector<idx>& parent, std::vector<idx>* sup_parent) {
  const idx ns = (idx)ptr.size() - 1;
  std::vector<idx> owner(ptr.empty() ? 0 : ptr.back());
  for (idx s = 0; s < ns; ++s)
    for (idx c = ptr[s]; c < ptr[s + 1]; ++c) owner[c] = s;
  sup_parent->assign(ns, -1);
  for (idx s = 0; s < ns; ++s) {
    const idx last = ptr[s + 1] - 1;
    if (parent[last] >= 0) (*sup_parent)[s] = owner[parent[last]];
  }
}

}  // namespace

int supernodal_analyze(const Pattern& p, const std::vector<idx>& perm, const std::vector<idx>& perm_inv,
                       idx max_child_size, double fill_tolerance, Supernodal* out) {
  const idx n = p.n;
  if ((idx)perm.size() != n || (idx)perm_inv.size() != n) return SP_BAD_SHAPE;
  {
    std::vector<char> seen(n, 0), seen2(n, 0);
    for (idx i = 0; i < n; ++i) {
      if (perm[i] < 0 || perm[i] >= n || seen[perm[i]]) return SP_BAD_SHAPE;
      if (perm_inv[i] < 0 || perm_inv[i] >= n || seen2[perm_inv[i]]) return SP_BAD_SHAPE;
      seen[perm[i]] = seen2[perm_inv[i]] = 1;
    }
  }
  Supernodal& S = *out;
  S.n = n;
  S.col_perm = perm;
  S.col_perm_inv = perm_inv;
  std::vector<size_t> tp, ti;
  transpose(p, &tp, &ti);
  col_etree(p, perm.data(), &S.etree);
  std::vector<idx> post;
  postorder(S.etree, &post);
  S.col_counts = counts_ata(n, tp, ti, perm_inv, S.etree, post);
  // fundamental supernodes: j extends the current one when it is the only
  // child's parent of j-1 and its count is one less
  if (n == 0) {
    S.supernode_ptr.assign(1, 0);
    S.super_etree.clear();
    return SP_OK;
  }
  std::vector<idx> nchild(n, 0);
  for (idx v = 0; v < n; ++v)
    if (S.etree[v] >= 0) nchild[S.etree[v]] += 1;
  std::vector<idx> sizes;
  sizes.push_back(1);
  for (idx j = 1; j < n; ++j) {
    const bool chain = S.etree[j - 1] == j && nchild[j] == 1 && S.col_counts[j - 1] == S.col_counts[j] + 1;
    if (chain)
      sizes.back() += 1;
    else
      sizes.push_back(1);
  }
  // relaxation: merge a small preceding supernode into the next one when the
  // zeros it adds stay within fill_tolerance of the expanded block
  const idx ns = (idx)sizes.size();
  std::vector<idx> fptr(ns + 1, 0);
  for (idx s = 0; s < ns; ++s) fptr[s + 1] = fptr[s] + sizes[s];
  std::vector<idx> deg(ns);
  for (idx s = 0; s < ns; ++s) deg[s] = std::max<idx>(S.col_counts[fptr[s + 1] - 1] - 1, 0);
  std::vector<char> alive(ns, 1);
  for (idx par = 1; par < ns; ++par) {
    const idx ch = par - 1;
    if (!alive[ch] || sizes[ch] > max_child_size) continue;
    const idx combined = sizes[par] + sizes[ch];
    const idx gain = std::max<idx>(deg[par] - deg[ch], 0);
    const idx extra = (sizes[par] + gain) * sizes[ch];
    const idx expanded = combined * (combined + 1) / 2 + deg[par] * combined;
    if ((double)extra <= fill_tolerance * (double)expanded) {
      sizes[par] = combined;
      alive[ch] = 0;
    }
  }
  S.supernode_ptr.assign(1, 0);
  for (idx s = 0; s < ns; ++s)
    if (alive[s]) S.supernode_ptr.push_back(S.supernode_ptr.back() + sizes[s]);
  tree_of_partition(S.supernode_ptr, S.etree, &S.super_etree);
  return SP_OK;
}

}  // namespace sp
}  // namespace alg
