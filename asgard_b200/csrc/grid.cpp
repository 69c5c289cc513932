// Host-side builder of the sparse-grid operator structure (setup, not timed).
//
// Re-creates what the reference builds before a kronmult_matrix exists:
//   * element table: level multi-indexes with |l|_1 <= L, grouped by level
//     sum from L down to 0, each group in lexicographic order with
//     dimension 0 fastest, each multi-index expanded to its cells with
//     dimension 0 fastest (src/elements.cpp:248-351,
//     src/permutations.hpp:71-180, src/elements.cpp:408-458);
//   * 1D connectivity: cells whose supports touch on the periodic unit
//     interval, per row in ascending order (connect_1d, full hierarchy,
//     src/asgard_grid_1d.hpp:19-330; a connection's index is its CSR
//     position, get_offset :92-122);
//   * connected cell pairs: connected in every dimension (check_connected,
//     src/asgard_kronmult_matrix.cpp:230-300), rows in table order and columns
//     ascending (make_kronmult_sparse, :406-466), with the d 1D connection
//     indices of each pair (compute_coefficient_offsets, :302-321).
#include "asgard_b200.h"

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <unordered_map>
#include <vector>

#include "internal.cuh"

#include <new>

#include <omp.h>

namespace
{
// (level, position) of a 1D hierarchical cell index
inline void split(int index, int &level, int &pos)
{
  if (index == 0)
  {
    level = 0;
    pos   = 0;
    return;
  }
  level = 32 - __builtin_clz(unsigned(index));
  pos   = index - (1 << (level - 1));
}

// Closed supports of (La, pa) and (Lb, pb) intersect on the periodic [0, 1].
bool supports_touch(int La, int pa, int Lb, int pb)
{
  if (La > Lb)
  {
    std::swap(La, Lb);
    std::swap(pa, pb);
  }
  if (La <= 1) // levels 0 and 1 cover the whole interval
    return true;
  int const lastA = (1 << (La - 1)) - 1, lastB = (1 << (Lb - 1)) - 1;
  if ((pa == 0 && pb == lastB) || (pb == 0 && pa == lastA))
    return true; // periodic wrap
  if (La == Lb)
    return std::abs(pa - pb) <= 1;
  // walk (Lb, pb) up to level La, tracking whether it stays on the left
  // (-1) or right (+1) edge of its ancestors
  int edge = (pb & 1) ? 1 : -1;
  while (Lb > La)
  {
    if (pb & 1)
      edge = (edge == 1) ? 1 : 0;
    else
      edge = (edge == -1) ? -1 : 0;
    pb >>= 1;
    --Lb;
  }
  return pb == pa || pb + edge == pa;
}

struct conn1d
{
  int rows = 0;
  std::vector<int> pntr, indx;
  std::vector<int> lut; // rows x rows, -1 when not connected
  explicit conn1d(int level)
  {
    rows = 1 << level;
    pntr.assign(rows + 1, 0);
    lut.assign(size_t(rows) * rows, -1);
    std::vector<int> la(rows), pa(rows);
    for (int i = 0; i < rows; i++)
      split(i, la[i], pa[i]);
    for (int r = 0; r < rows; r++)
    {
      for (int c = 0; c < rows; c++)
        if (supports_touch(la[r], pa[r], la[c], pa[c]))
        {
          lut[size_t(r) * rows + c] = int(indx.size());
          indx.push_back(c);
        }
      pntr[r + 1] = int(indx.size());
    }
  }
};

inline int index_1d(int level, int pos)
{
  return level == 0 ? 0 : (1 << (level - 1)) + pos;
}

} // namespace

namespace asgk
{
// Neighbours of every cell along one dimension at a time: cell c is listed
// for row r and dimension k when c agrees with r in every other dimension
// and the 1D cells of r and c in dimension k are connected (c == r, with
// the self-connection, for every k).  These are the cell pairs of the
// connected-pair list that differ in at most one dimension -- the only
// pairs a term acting in a single dimension couples.
int build_direction_pairs(int d, int level, int num_cells, const int *table,
                          direction_pairs &out)
{
  if (d < 1 || d > 6 || level < 0 || level > 12 || num_cells < 0 || !table)
    return ASGK_ERR_INVALID;
  conn1d const c(level);
  int const R = c.rows;
  std::vector<int> oned(size_t(num_cells) * d);
  for (int i = 0; i < num_cells; i++)
    for (int k = 0; k < d; k++)
    {
      int const L = table[int64_t(i) * 2 * d + k];
      int const p = table[int64_t(i) * 2 * d + d + k];
      if (L < 0 || L > level || p < 0 || (L > 1 && p >= (1 << (L - 1))) ||
          (L <= 1 && p != 0))
        return ASGK_ERR_INVALID;
      oned[size_t(i) * d + k] = index_1d(L, p);
    }
  // 1D-index tuple -> cell (1D indices < 2^level: level bits each)
  int const bits = std::max(level, 1);
  if (d * bits > 64)
    return ASGK_ERR_UNSUPPORTED;
  auto key = [&](const int *t) {
    uint64_t h = 0;
    for (int k = 0; k < d; k++)
      h = (h << bits) | uint64_t(t[k]);
    return h;
  };
  std::unordered_map<uint64_t, int> where;
  where.reserve(size_t(num_cells) * 2);
  for (int i = 0; i < num_cells; i++)
    if (!where.emplace(key(&oned[size_t(i) * d]), i).second)
      return ASGK_ERR_INVALID; // a cell listed twice
  out.d = d;
  out.ptr.assign(num_cells + 1, 0);
  out.col.clear();
  out.dim.clear();
  out.conn.clear();
  out.self_conn.assign(size_t(num_cells) * d, -1);
  std::vector<int> t(d);
  for (int r = 0; r < num_cells; r++)
  {
    const int *ro = &oned[size_t(r) * d];
    for (int k = 0; k < d; k++)
    {
      std::copy(ro, ro + d, t.begin());
      int const rk = ro[k];
      for (int j = c.pntr[rk]; j < c.pntr[rk + 1]; j++)
      {
        t[k]          = c.indx[j];
        auto const it = where.find(key(t.data()));
        if (it == where.end())
          continue;
        out.col.push_back(it->second);
        out.dim.push_back(k);
        out.conn.push_back(j);
        if (it->second == r)
          out.self_conn[size_t(r) * d + k] = j;
      }
    }
    out.ptr[r + 1] = int64_t(out.col.size());
  }
  out.nconn = int(c.indx.size());
  out.conn_row.resize(c.indx.size());
  out.conn_col = c.indx;
  for (int r = 0; r < R; r++)
    for (int j = c.pntr[r]; j < c.pntr[r + 1]; j++)
      out.conn_row[j] = r;
  return ASGK_OK;
}
} // namespace asgk

extern "C"
{
int asgk_connect_1d(int level, int *num_rows, int *num_conn, int *pntr,
                    int *indx)
{
  try
  {
    if (level < 0 || level > 12 || !num_rows || !num_conn)
      return ASGK_ERR_INVALID;
    conn1d c(level);
    *num_rows = c.rows;
    *num_conn = int(c.indx.size());
    if (pntr)
      std::copy(c.pntr.begin(), c.pntr.end(), pntr);
    if (indx)
      std::copy(c.indx.begin(), c.indx.end(), indx);
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int64_t asgk_sparse_grid(int d, int level, int *table)
{
  if (d < 1 || d > 6 || level < 0 || level > 20)
    return -1;
  int64_t count = 0;
  for (int sum = level; sum >= 0; --sum)
  {
    int lv[6] = {0, 0, 0, 0, 0, 0};
    for (;;)
    {
      int tot = 0;
      for (int k = 0; k < d; k++)
        tot += lv[k];
      if (tot == sum)
      {
        int64_t cells = 1;
        int lim[6];
        for (int k = 0; k < d; k++)
        {
          lim[k] = lv[k] <= 1 ? 1 : (1 << (lv[k] - 1));
          cells *= lim[k];
        }
        if (table)
        {
          int pos[6] = {0, 0, 0, 0, 0, 0};
          for (int64_t c = 0; c < cells; c++)
          {
            int *row = table + (count + c) * 2 * d;
            for (int k = 0; k < d; k++)
            {
              row[k]     = lv[k];
              row[d + k] = pos[k];
            }
            for (int k = 0; k < d; k++) // dimension 0 fastest
            {
              if (++pos[k] < lim[k])
                break;
              pos[k] = 0;
            }
          }
        }
        count += cells;
      }
      // next multi-index (dimension 0 fastest) whose entries sum to <= sum
      int k = 0;
      for (; k < d; k++)
      {
        lv[k]++;
        int t = 0;
        for (int q = 0; q < d; q++)
          t += lv[q];
        if (t <= sum)
          break;
        lv[k] = 0;
      }
      if (k == d)
        break;
    }
  }
  return count;
}

int asgk_build_pairs(int d, int level, int num_cells, const int *table,
                     int64_t *nnz, int64_t *row_ptr, int *col_indx, int *conn)
{
  try
  {
    if (d < 1 || d > 6 || level < 0 || level > 12 || num_cells < 0 || !table ||
        !nnz)
      return ASGK_ERR_INVALID;
    conn1d const c(level);
    int const R = c.rows;
    // per cell: its 1D index in every dimension
    std::vector<int> oned(size_t(num_cells) * d);
    for (int i = 0; i < num_cells; i++)
      for (int k = 0; k < d; k++)
      {
        int const L = table[int64_t(i) * 2 * d + k];
        int const p = table[int64_t(i) * 2 * d + d + k];
        if (L < 0 || L > level || p < 0 || (L > 1 && p >= (1 << (L - 1))) ||
            (L <= 1 && p != 0))
          return ASGK_ERR_INVALID;
        oned[size_t(i) * d + k] = index_1d(L, p);
      }
    std::vector<int64_t> counts(num_cells, 0);
  #pragma omp parallel for schedule(dynamic, 16)
    for (int r = 0; r < num_cells; r++)
    {
      const int *ro = &oned[size_t(r) * d];
      int64_t cnt   = 0;
      for (int cc = 0; cc < num_cells; cc++)
      {
        const int *co = &oned[size_t(cc) * d];
        bool ok       = true;
        for (int k = 0; k < d && ok; k++)
          ok = c.lut[size_t(ro[k]) * R + co[k]] >= 0;
        cnt += ok;
      }
      counts[r] = cnt;
    }
    int64_t total = 0;
    for (int r = 0; r < num_cells; r++)
      total += counts[r];
    *nnz = total;
    if (!row_ptr || !col_indx)
      return ASGK_OK;
    row_ptr[0] = 0;
    for (int r = 0; r < num_cells; r++)
      row_ptr[r + 1] = row_ptr[r] + counts[r];
  #pragma omp parallel for schedule(dynamic, 16)
    for (int r = 0; r < num_cells; r++)
    {
      const int *ro = &oned[size_t(r) * d];
      int64_t pos   = row_ptr[r];
      for (int cc = 0; cc < num_cells; cc++)
      {
        const int *co = &oned[size_t(cc) * d];
        int off[6];
        bool ok = true;
        for (int k = 0; k < d && ok; k++)
        {
          off[k] = c.lut[size_t(ro[k]) * R + co[k]];
          ok     = off[k] >= 0;
        }
        if (!ok)
          continue;
        col_indx[pos] = cc;
        if (conn)
          for (int k = 0; k < d; k++)
            conn[pos * d + k] = off[k];
        ++pos;
      }
    }
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

int asgk_direction_pairs(int d, int level, int num_cells, const int *table,
                         int64_t *nnz, int64_t *row_ptr, int *col_indx,
                         int *dim, int *conn)
{
  try
  {
    if (!nnz)
      return ASGK_ERR_INVALID;
    asgk::direction_pairs dp;
    if (int rc = asgk::build_direction_pairs(d, level, num_cells, table, dp))
      return rc;
    *nnz = int64_t(dp.col.size());
    if (row_ptr)
      std::copy(dp.ptr.begin(), dp.ptr.end(), row_ptr);
    if (col_indx)
      std::copy(dp.col.begin(), dp.col.end(), col_indx);
    if (dim)
      std::copy(dp.dim.begin(), dp.dim.end(), dim);
    if (conn)
      std::copy(dp.conn.begin(), dp.conn.end(), conn);
    return ASGK_OK;
  }
  catch (std::bad_alloc const &)
  {
    return ASGK_ERR_ALLOC;
  }
  catch (...)
  {
    return ASGK_ERR_INVALID;
  }
}

} // extern "C"
