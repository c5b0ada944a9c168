// Rasterisation rules shared by the host rasteriser and the device kernels.
//
// A parsed geometry becomes a plan in pixel space (grid columns and rows,
// through the inverse geo transform): points and line segments as runs of
// samples, polygons as edge lists over a range of rows.  The sequential
// execution on the host (run_plan_host below) and the kernels of raster.cu
// call the same per-sample and per-edge functions, so both burn the same
// cells.  The rules are GDALRasterizeGeometries' default (not all-touched)
// burning, which the reference's rasterize_times and rasterize_fuels use
// (crates/propag/src/propag.rs:837-890, 929-982):
//   * a point burns the cell that holds it;
//   * a segment p0 -> p1 takes steps = ceil(max(|dcol|, |drow|)) equal steps
//     and burns the cell under each sample p0 + (s / steps) (p1 - p0),
//     s = 0 .. steps;
//   * a polygon burns the cells whose centre lies inside it, by the even-odd
//     rule over all of its rings (each ring closed): on the centre line
//     y = row + 0.5 an edge crosses when its ends straddle y half-open
//     (y0 <= y < y1), and the cells inside are those with an odd number of
//     crossings x at or left of their centre (x - 0.5 <= col).
// Features burn in order, so where several cover a cell the last one wins.
//
// Pixel arithmetic is plain IEEE double (no contraction: the device file is
// compiled with -fmad=false, the host one as ISO C++ without FMA), so both
// executions round identically.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <vector>

#if defined(__CUDACC__)
#define PG_HD __host__ __device__
#else
#define PG_HD
#endif

namespace propag {

struct Pt {
  double x, y;
};

// A point or one segment of a line, in pixel space.
struct RasterSeg {
  double c0, r0;    // first sample (column, row)
  double dc, dr;    // p1 - p0
  double steps;     // an integer; 0 for a point
  int64_t s0, s1;   // the samples that can land in the grid, s0 <= s1
  uint64_t before;  // samples of the segments ahead of this one in the plan
  int32_t feature;
  int32_t pad_;
};

// One polygon edge in pixel space.
struct RasterEdge {
  double ax, ay, bx, by;
};

// A polygon: edges [first, first + count) and grid rows [row0, row1].
struct RasterPoly {
  uint64_t first;
  uint64_t before;  // rows of the polygons ahead of this one in the plan
  uint32_t count;
  int32_t feature;
  int32_t row0, row1;
};

// Segments and polygons that reach a W x H grid, in burn order.
struct RasterPlan {
  std::vector<RasterSeg> segs;
  std::vector<RasterEdge> edges;
  std::vector<RasterPoly> polys;
  uint64_t samples = 0;  // sum over segs of s1 - s0 + 1
  uint64_t rows = 0;     // sum over polys of row1 - row0 + 1
};

// A plan's arrays in device memory.
struct RasterPlanDev {
  const RasterSeg *segs;
  uint64_t nseg, samples;
  const RasterPoly *polys;
  uint64_t npoly, rows;
  const RasterEdge *edges;
};

// Lines whose ends lie further than this many cells from the origin are left
// out (their sampling would not be exact in double precision).
constexpr double kRasterMaxCoord = 1099511627776.0;  // 2^40

// floor(v) as an index into [0, n), or -1 (NaN included).
PG_HD inline int64_t cell_of(double v, int64_t n) {
  const double f = floor(v);
  return (f >= 0.0 && f < (double)n) ? (int64_t)f : -1;
}

// The cell under sample s of segment g; false when it is outside the grid.
PG_HD inline bool seg_sample(const RasterSeg &g, int64_t s, int64_t W, int64_t H, int64_t &c,
                             int64_t &r) {
  double x = g.c0, y = g.r0;
  if (g.steps > 0.0) {
    const double t = (double)s / g.steps;
    x = g.c0 + t * g.dc;
    y = g.r0 + t * g.dr;
  }
  c = cell_of(x, W);
  r = cell_of(y, H);
  return c >= 0 && r >= 0;
}

// Where edge e crosses the centre line y = yc, if it does.
PG_HD inline bool edge_crossing(const RasterEdge &e, double yc, double &x) {
  if ((e.ay <= yc && e.by > yc) || (e.by <= yc && e.ay > yc)) {
    x = e.ax + (yc - e.ay) * (e.bx - e.ax) / (e.by - e.ay);
    return true;
  }
  return false;
}

// The first column whose centre lies at or right of crossing x,
// ceil(x - 0.5), raised to 0; W when no column of the row does.
PG_HD inline int64_t crossing_cell(double x, int64_t W) {
  const double t = ceil(x - 0.5);
  if (!(t < (double)W)) return W;
  return t < 0.0 ? 0 : (int64_t)t;
}

// Appends a point (c1, r1 = c0, r0) or a line segment of feature `feature`,
// in pixel space, to the plan; one that misses the W x H grid is dropped.
inline void plan_segment(RasterPlan &plan, double c0, double r0, double c1, double r1,
                         int32_t feature, int64_t W, int64_t H) {
  const double lim = kRasterMaxCoord;
  if (!(std::fabs(c0) <= lim && std::fabs(r0) <= lim && std::fabs(c1) <= lim &&
        std::fabs(r1) <= lim))
    return;
  RasterSeg g{};
  g.c0 = c0;
  g.r0 = r0;
  g.dc = c1 - c0;
  g.dr = r1 - r0;
  g.steps = std::ceil(std::max(std::fabs(g.dc), std::fabs(g.dr)));
  g.feature = feature;
  double lo = 0.0, hi = g.steps;
  // Samples whose column (row) can fall inside [0, n): the exact position
  // p0 + s d / steps must lie in (-1, n + 1), the rounded one being within a
  // small fraction of a cell of it; two samples of margin on each side.
  auto clip = [&](double p0, double d, double n) {
    if (d == 0.0) {
      if (!(p0 > -1.0 && p0 < n + 1.0)) hi = -1.0;
      return;
    }
    double a = (-1.0 - p0) / d * g.steps, b = (n + 1.0 - p0) / d * g.steps;
    if (a > b) std::swap(a, b);
    lo = std::max(lo, std::floor(a) - 2.0);
    hi = std::min(hi, std::ceil(b) + 2.0);
  };
  if (g.steps > 0.0) {
    clip(c0, g.dc, (double)W);
    clip(r0, g.dr, (double)H);
  }
  if (!(lo <= hi)) return;
  g.s0 = (int64_t)lo;
  g.s1 = (int64_t)hi;
  if (g.steps == 0.0) {  // a point: keep it only when it lands in the grid
    int64_t c, r;
    if (!seg_sample(g, 0, W, H, c, r)) return;
  }
  g.before = plan.samples;
  plan.samples += (uint64_t)(g.s1 - g.s0 + 1);
  plan.segs.push_back(g);
}

// A polygon of rings in pixel space; a ring whose ends differ is closed.
inline void plan_polygon(RasterPlan &plan, const std::vector<std::vector<Pt>> &rings,
                         int32_t feature, int64_t H) {
  RasterPoly p{};
  p.first = plan.edges.size();
  p.feature = feature;
  double rmin = 1e300, rmax = -1e300;
  for (const auto &ring : rings) {
    for (const Pt &q : ring) {
      rmin = std::min(rmin, q.y);
      rmax = std::max(rmax, q.y);
    }
    for (size_t k = 0; k + 1 < ring.size(); ++k)
      plan.edges.push_back({ring[k].x, ring[k].y, ring[k + 1].x, ring[k + 1].y});
    if (ring.size() >= 2 && (ring.front().x != ring.back().x || ring.front().y != ring.back().y))
      plan.edges.push_back({ring.back().x, ring.back().y, ring.front().x, ring.front().y});
  }
  const uint64_t count = plan.edges.size() - p.first;
  const double r0 = std::max(0.0, std::floor(rmin)), r1 = std::min((double)H - 1.0, std::ceil(rmax));
  if (count == 0 || count > 0xFFFFFFFFull || !(r0 <= r1)) {
    plan.edges.resize(p.first);
    return;
  }
  p.count = (uint32_t)count;
  p.row0 = (int32_t)r0;
  p.row1 = (int32_t)r1;
  p.before = plan.rows;
  plan.rows += (uint64_t)(p.row1 - p.row0 + 1);
  plan.polys.push_back(p);
}

// Sequential execution of a plan: burn(feature, col, row) for every cell, in
// plan order (segments, then polygons row by row, columns ascending).
template <typename F>
void run_plan_host(const RasterPlan &plan, int64_t W, int64_t H, F &&burn) {
  for (const RasterSeg &g : plan.segs)
    for (int64_t s = g.s0; s <= g.s1; ++s) {
      int64_t c, r;
      if (seg_sample(g, s, W, H, c, r)) burn(g.feature, c, r);
    }
  std::vector<int64_t> cut;
  for (const RasterPoly &p : plan.polys)
    for (int64_t r = p.row0; r <= p.row1; ++r) {
      const double yc = (double)r + 0.5;
      cut.clear();
      for (uint64_t k = 0; k < p.count; ++k) {
        double x;
        if (!edge_crossing(plan.edges[p.first + k], yc, x)) continue;
        const int64_t c = crossing_cell(x, W);
        if (c < W) cut.push_back(c);
      }
      std::sort(cut.begin(), cut.end());
      // odd counts of crossings at or left of a cell: [cut0, cut1), [cut2, cut3), ...
      for (size_t k = 0; k < cut.size(); k += 2) {
        const int64_t end = k + 1 < cut.size() ? cut[k + 1] : W;
        for (int64_t c = cut[k]; c < end; ++c) burn(p.feature, c, r);
      }
    }
}

}  // namespace propag
