// ipg_snap_tables.cu — host construction of the SNAP index and Clebsch–Gordan tables.
//
// The tables are those of initialize_prebuilt_arrays
// (src/BasisSystems/SNAP/types/prebuilt_arrays.jl:48-321): the same enumeration order of
// (j1 >= j2, j = |j1-j2|..min(J, j1+j2) step 2) blocks, the same CG coefficients (factorial
// sums, :250-312) and sqrt(p/q) roots (:314-321), because the descriptors are defined by
// that ordering.  Derived tables (half-plane offsets, the Y gather list, the dB term list)
// are new and serve the CUDA kernels.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "ipg_snap.cuh"

namespace {

// Factorials as long double (64-bit mantissa): exact wherever the reference's Int64
// products are exact (twojmax <= 8), and free of Int64 overflow beyond that.
long double fact(int n) {
  long double f = 1.0L;
  for (int k = 2; k <= n; k++) f *= k;
  return f;
}

// prebuilt_arrays.jl:250-257
double delta_cg(int j1, int j2, int j) {
  long double den = fact((j1 + j2 + j) / 2 + 1);
  long double num = fact((j1 + j2 - j) / 2) * fact((j1 - j2 + j) / 2) * fact((-j1 + j2 + j) / 2);
  return std::sqrt((double)num / (double)den);
}

}  // namespace

int snap_build_tables(const ipg_snap_params& p, SnapHost& h) {
  const int J = p.twojmax;
  if (J < 0 || J > SNAP_MAX_J) return IPG_ERR_ARG;
  const int jd = J + 1;
  h.J = J;
  auto blk = [jd](int a, int b, int c) { return (a * jd + b) * jd + c; };
  h.idxcg_block.assign(jd * jd * jd, -1);
  h.idxz_block.assign(jd * jd * jd, -1);
  h.idxb_block.assign(jd * jd * jd, -1);
  h.idxu_block.assign(jd, 0);
  h.half_block.assign(jd + 1, 0);

  int cnt = 0;
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
        h.idxcg_block[blk(j1, j2, j)] = cnt;
        cnt += (j1 + 1) * (j2 + 1);
      }
  h.idxcg_max = cnt;

  cnt = 0;
  for (int j = 0; j <= J; j++) {
    h.idxu_block[j] = cnt;
    cnt += (j + 1) * (j + 1);
  }
  h.idxu_max = cnt;

  // half plane: rows mb = 0..j/2 of every level
  cnt = 0;
  h.ext_max = 1;
  for (int j = 0; j <= J; j++) {
    h.half_block[j] = cnt;
    cnt += (j / 2 + 1) * (j + 1);
    h.ext_max = std::max(h.ext_max, ((j + 1) / 2 + 1) * (j + 1));
  }
  h.half_block[jd] = cnt;
  h.u_half = cnt;
  h.h_info.clear();
  h.h_sgen.clear();
  for (int j = 0; j <= J; j++)
    for (int mb = 0; 2 * mb <= j; mb++)
      for (int m = 0; m <= j; m++) {
        const int last = (2 * mb == j) ? mb : j;  // the middle row of an even level is weighted up to mb
        h.h_info.push_back(m | (j << 8) | ((m <= last ? 1 : 0) << 16));
        h.h_sgen.push_back(m < j ? std::sqrt((double)((m + 1) * (j - m))) : 0.0);
        h.h_sgen.push_back(m >= 1 ? std::sqrt((double)(m * (j - m + 1))) : 0.0);
      }

  h.idxb.clear();
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2)
        if (j >= j1) {
          h.idxb_block[blk(j1, j2, j)] = (int)h.idxb.size() / 3;
          h.idxb.push_back(j1);
          h.idxb.push_back(j2);
          h.idxb.push_back(j);
        }
  h.idxb_max = (int)h.idxb.size() / 3;

  h.idxz.clear();
  h.zjju_half.clear();
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
        h.idxz_block[blk(j1, j2, j)] = (int)h.idxz.size();
        for (int mb = 0; 2 * mb <= j; mb++)
          for (int ma = 0; ma <= j; ma++) {
            int ma1min = std::max(0, (2 * ma - j - j2 + j1) / 2);
            int ma2max = (2 * ma - j - (2 * ma1min - j1) + j2) / 2;
            int na = std::min(j1, (2 * ma - j + j2 + j1) / 2) - ma1min + 1;
            int mb1min = std::max(0, (2 * mb - j - j2 + j1) / 2);
            int mb2max = (2 * mb - j - (2 * mb1min - j1) + j2) / 2;
            int nb = std::min(j1, (2 * mb - j + j2 + j1) / 2) - mb1min + 1;
            ZDev z;
            z.j1 = (int8_t)j1;
            z.j2 = (int8_t)j2;
            z.j = (int8_t)j;
            z.na = (int8_t)na;
            z.nb = (int8_t)nb;
            z.pad0 = z.pad1 = z.pad2 = 0;
            z.ma1min = (int8_t)ma1min;
            z.ma2max = (int8_t)ma2max;
            z.mb1min = (int8_t)mb1min;
            z.mb2max = (int8_t)mb2max;
            z.u1base = h.idxu_block[j1] + (j1 + 1) * mb1min + ma1min;
            z.u2base = h.idxu_block[j2] + (j2 + 1) * mb2max + ma2max;
            z.icga0 = ma1min * (j2 + 1) + ma2max;
            z.icgb0 = mb1min * (j2 + 1) + mb2max;
            z.cgoff = h.idxcg_block[blk(j1, j2, j)];
            h.idxz.push_back(z);
            h.zjju_half.push_back(h.half_block[j] + (j + 1) * mb + ma);
          }
      }
  h.idxz_max = (int)h.idxz.size();

  h.rootpq.assign((J + 2) * (J + 2), 0.0);
  for (int a = 1; a <= J; a++)
    for (int b = 1; b <= J; b++) h.rootpq[a * (J + 2) + b] = std::sqrt((double)a / (double)b);

  h.cglist.assign(h.idxcg_max, 0.0);
  int idx = 0;
  for (int j1 = 0; j1 <= J; j1++)
    for (int j2 = 0; j2 <= j1; j2++)
      for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2)
        for (int m1 = 0; m1 <= j1; m1++) {
          int aa2 = 2 * m1 - j1;
          for (int m2 = 0; m2 <= j2; m2++, idx++) {
            int bb2 = 2 * m2 - j2;
            int m = (aa2 + bb2 + j) / 2;
            if (m < 0 || m > j) continue;
            double sum = 0.0;
            int zmin = std::max(0, std::max(-(j - j2 + aa2) / 2, -(j - j1 - bb2) / 2));
            int zmax = std::min((j1 + j2 - j) / 2, std::min((j1 - aa2) / 2, (j2 + bb2) / 2));
            for (int z = zmin; z <= zmax; z++) {
              long double den = fact(z) * fact((j1 + j2 - j) / 2 - z) * fact((j1 - aa2) / 2 - z) * fact((j2 + bb2) / 2 - z) *
                            fact((j - j2 + aa2) / 2 + z) * fact((j - j1 - bb2) / 2 + z);
              sum += ((z % 2 == 0) ? 1.0 : -1.0) / (double)den;
            }
            int cc2 = 2 * m - j;
            long double sf = fact((j1 + aa2) / 2) * fact((j1 - aa2) / 2) * fact((j2 + bb2) / 2) * fact((j2 - bb2) / 2) *
                         fact((j + cc2) / 2) * fact((j - cc2) / 2) * (long double)(j + 1);
            h.cglist[idx] = sum * delta_cg(j1, j2, j) * std::sqrt((double)sf);
          }
        }

  // bzero (prebuilt_arrays.jl:52-63); wself = 1
  h.bzero.assign(jd, 0.0);
  if (p.bzero_flag)
    for (int j = 0; j <= J; j++) h.bzero[j] = p.bnorm_flag ? 1.0 : (double)(j + 1);

  // dB terms (compute_b.jl:207-400): Z(j1,j2,j) on level j, (j+1)/(j1+1) Z(j,j2,j1) on
  // level j1, (j+1)/(j2+1) Z(j,j1,j2) on level j2 (factors dropped when bnorm_flag).
  h.db.resize(h.idxb_max);
  for (int b = 0; b < h.idxb_max; b++) {
    int j1 = h.idxb[3 * b], j2 = h.idxb[3 * b + 1], j = h.idxb[3 * b + 2];
    DBDev& d = h.db[b];
    d.l[0] = j;
    d.z0[0] = h.idxz_block[blk(j1, j2, j)];
    d.fac[0] = 1.0;
    d.l[1] = j1;
    d.z0[1] = h.idxz_block[blk(j, j2, j1)];
    d.fac[1] = p.bnorm_flag ? 1.0 : (j + 1) / (j1 + 1.0);
    d.l[2] = j2;
    d.z0[2] = h.idxz_block[blk(j, j1, j2)];
    d.fac[2] = p.bnorm_flag ? 1.0 : (j + 1) / (j2 + 1.0);
  }

  // Y = d(beta . B)/dU (design of compute_yi.jl:86-118): each Z entry (J1,J2,J,ma,mb)
  // feeds Y(J,ma,mb) with weight beta[jjb] times multiplicity and (J1+1)/(J+1).
  h.y_jjb.assign(h.idxz_max, 0);
  h.y_mult.assign(h.idxz_max, 0.0);
  for (int z = 0; z < h.idxz_max; z++) {
    int j1 = h.idxz[z].j1, j2 = h.idxz[z].j2, j = h.idxz[z].j;
    int jjb;
    double mult;
    if (j >= j1) {
      jjb = h.idxb_block[blk(j1, j2, j)];
      mult = (j1 == j) ? ((j2 == j) ? 3.0 : 2.0) : 1.0;
    } else if (j >= j2) {
      jjb = h.idxb_block[blk(j, j2, j1)];
      mult = (j2 == j) ? 2.0 : 1.0;
    } else {
      jjb = h.idxb_block[blk(j2, j, j1)];
      mult = 1.0;
    }
    if (!p.bnorm_flag && j1 > j) mult *= (j1 + 1) / (j + 1.0);
    h.y_jjb[z] = jjb;
    h.y_mult[z] = mult;
  }
  h.y_off.assign(h.u_half + 1, 0);
  for (int z = 0; z < h.idxz_max; z++) h.y_off[h.zjju_half[z] + 1]++;
  for (int q = 0; q < h.u_half; q++) h.y_off[q + 1] += h.y_off[q];
  // Z entries in order of their loop shape, so that the threads of a warp that take
  // consecutive entries run identical (nb, na) trip counts
  h.zperm.resize(h.idxz_max);
  for (int z = 0; z < h.idxz_max; z++) h.zperm[z] = z;
  std::stable_sort(h.zperm.begin(), h.zperm.end(), [&](int a, int b) {
    const ZDev &p = h.idxz[a], &q = h.idxz[b];
    return p.nb != q.nb ? p.nb < q.nb : p.na < q.na;
  });
  // Y schedule: every half-plane entry with nonzero weight goes to one of YS_WARPS warps,
  // longest first to the least loaded warp (cost = inner terms of its Z entries)
  {
    h.u_of_h.assign(h.u_half, 0);
    std::vector<std::pair<double, int>> cost;  // (cost, h)
    std::vector<double> wgt(h.u_half, 0.0);
    std::vector<double> hc(h.u_half, 0.0);
    for (int z = 0; z < h.idxz_max; z++) hc[h.zjju_half[z]] += h.idxz[z].nb * (2.0 + h.idxz[z].na) + 2.0;
    for (int j = 0; j <= J; j++)
      for (int mb = 0; 2 * mb <= j; mb++)
        for (int ma = 0; ma <= j; ma++) {
          const int hh = h.half_block[j] + mb * (j + 1) + ma;
          h.u_of_h[hh] = h.idxu_block[j] + mb * (j + 1) + ma;
          wgt[hh] = (2 * mb < j) ? 1.0 : (ma < mb ? 1.0 : (ma == mb ? 0.5 : 0.0));
          if (wgt[hh] != 0.0) cost.push_back({hc[hh], hh});
        }
    std::stable_sort(cost.begin(), cost.end(), [](const std::pair<double, int>& a, const std::pair<double, int>& b) {
      return a.first > b.first;
    });
    std::vector<std::vector<int>> bins(YS_WARPS);
    std::vector<double> load(YS_WARPS, 0.0);
    for (auto& c : cost) {
      int w = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      bins[w].push_back(c.second);
      load[w] += c.first;
    }
    h.ysched_off.assign(YS_WARPS + 1, 0);
    h.ysched_h.clear();
    h.ysched_w.clear();
    for (int w = 0; w < YS_WARPS; w++) {
      std::sort(bins[w].begin(), bins[w].end());
      for (int hh : bins[w]) {
        h.ysched_h.push_back(hh);
        h.ysched_w.push_back(wgt[hh]);
      }
      h.ysched_off[w + 1] = (int)h.ysched_h.size();
    }
  }
  h.y_jjz.assign(h.idxz_max, 0);
  std::vector<int32_t> fill(h.y_off.begin(), h.y_off.end() - 1);
  for (int z = 0; z < h.idxz_max; z++) h.y_jjz[fill[h.zjju_half[z]]++] = z;

  // Row-blocked Y schedule.  Target row (j, mb) of the half plane collects, for every
  // triple (j1 >= j2, j), the Z entries (j1, j2, j, ma, mb) of all ma at once: the nb row
  // pairs (mb1, mb2) are the same for every ma, and for one row pair
  //   Z(ma) += cg[mb1][mb2] sum_ma2 cg[ma + d - ma2][ma2] U(j1, mb1, ma + d - ma2) U(j2, mb2, ma2)
  // with d = (j1 + j2 - j)/2.  The CG factors ca[ma][ma2] of a triple are stored by column
  // pair as [m0/2][ma][2] (yca; 16-byte pairs), zero where ma2 > j2 or ma1 = ma + d - ma2
  // falls outside 0..j1.  Rows are listed longest first (the kernel hands them out in
  // that order to whichever warp is free).
  h.yrows.clear();
  h.yitems.clear();
  h.yca.clear();
  h.ytrip_jjz.clear();
  if (J <= YR_MAX_J) {
    std::vector<int32_t> ca_of(jd * jd * jd, -1), trip_of(jd * jd * jd, -1);
    for (int j1 = 0; j1 <= J; j1++)
      for (int j2 = 0; j2 <= j1; j2++)
        for (int j = j1 - j2; j <= std::min(J, j1 + j2); j += 2) {
          const int d = (j1 + j2 - j) / 2, cg0 = h.idxcg_block[blk(j1, j2, j)];
          ca_of[blk(j1, j2, j)] = (int32_t)h.yca.size();
          trip_of[blk(j1, j2, j)] = (int32_t)h.ytrip_jjz.size();
          h.ytrip_jjz.push_back(h.idxz_block[blk(j1, j2, j)]);
          for (int m0 = 0; m0 <= j2; m0 += 2)  // column pairs (m0, m0 + 1), as [m0/2][ma][2]
            for (int ma = 0; ma <= j; ma++)
              for (int q = 0; q < 2; q++) {
                const int ma2 = m0 + q, ma1 = ma + d - ma2;
                const bool ok = ma2 <= j2 && ma1 >= 0 && ma1 <= j1;
                h.yca.push_back(ok ? h.cglist[cg0 + ma1 * (j2 + 1) + ma2] : 0.0);
              }
        }
    struct Row {
      YRowDev r;
      std::vector<YItemDev> items;
      double cost;
    };
    std::vector<Row> rows;
    for (int j = 0; j <= J; j++)
      for (int mb = 0; 2 * mb <= j; mb++) {
        Row row;
        row.r.j = (int8_t)j;
        row.r.mb = (int8_t)mb;
        row.r.mid = (int8_t)(2 * mb == j);
        row.r.pad = 0;
        row.r.h0 = h.half_block[j] + mb * (j + 1);
        row.cost = 0.0;
        const int nma = row.r.mid ? mb + 1 : j + 1;
        for (int j1 = 0; j1 <= J; j1++)
          for (int j2 = 0; j2 <= j1; j2++) {
            if (j < j1 - j2 || j > std::min(J, j1 + j2) || ((j1 + j2 + j) & 1)) continue;
            const int mb1min = std::max(0, (2 * mb - j - j2 + j1) / 2);
            const int mb2max = (2 * mb - j - (2 * mb1min - j1) + j2) / 2;
            const int nb = std::min(j1, (2 * mb - j + j2 + j1) / 2) - mb1min + 1;
            if (nb <= 0) continue;
            YItemDev it;
            it.j1 = (int8_t)j1;
            it.j2 = (int8_t)j2;
            it.d = (int8_t)((j1 + j2 - j) / 2);
            it.nb = (int8_t)nb;
            it.mb1min = (int8_t)mb1min;
            it.mb2max = (int8_t)mb2max;
            it.pad0 = it.pad1 = 0;
            it.ca = ca_of[blk(j1, j2, j)];
            it.cg = h.idxcg_block[blk(j1, j2, j)];
            it.jjz = h.idxz_block[blk(j1, j2, j)];
            it.trip = trip_of[blk(j1, j2, j)];
            row.items.push_back(it);
            row.cost += nb * (6.0 * nma * (j2 + 1) + (nma + 2 * j2 + 8));
          }
        rows.push_back(row);
      }
    std::vector<int> order(rows.size());
    for (size_t q = 0; q < rows.size(); q++) order[q] = (int)q;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return rows[a].cost > rows[b].cost; });
    for (int q : order) {
      YRowDev r = rows[q].r;
      r.t0 = (int32_t)h.yitems.size();
      h.yitems.insert(h.yitems.end(), rows[q].items.begin(), rows[q].items.end());
      r.t1 = (int32_t)h.yitems.size();
      h.yrows.push_back(r);
    }
    // the constant-bank copy: item.cg becomes the offset of its first row factor in cb
    memset(&h.yconst, 0, sizeof(h.yconst));
    int nrp = 0;
    for (const YItemDev& it : h.yitems) nrp += it.nb;
    h.yconst_ok = (int)h.yrows.size() <= YC_ROWS && (int)h.yitems.size() <= YC_ITEMS && nrp <= YC_RP;
    if (h.yconst_ok) {
      YConst& C = h.yconst;
      C.nrows = (int)h.yrows.size();
      C.nitems = (int)h.yitems.size();
      for (int q = 0; q < C.nrows; q++) C.rows[q] = h.yrows[q];
      int o = 0;
      for (int t = 0; t < C.nitems; t++) {
        YItemDev it = h.yitems[t];
        const int cg0 = it.cg;
        it.cg = o;
        for (int ib = 0; ib < it.nb; ib++)
          C.cb[o++] = h.cglist[cg0 + (it.mb1min + ib) * (it.j2 + 1) + (it.mb2max - ib)];
        C.items[t] = it;
      }
      C.nrp = o;
    }
  }
  return IPG_OK;
}
