// GDAL-free geometry and raster I/O used by the plugin ABI.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "propag_host.h"

namespace propag {

struct Pt {
  double x, y;
};

// One parsed WKB geometry flattened into its parts.
struct Geometry {
  std::vector<Pt> points;                       // Point / MultiPoint
  std::vector<std::vector<Pt>> lines;           // LineString / MultiLineString
  std::vector<std::vector<std::vector<Pt>>> polygons;  // Polygon rings
};

// Parses ISO / EWKB (2D, Z, M, ZM, either byte order).  Returns false on
// malformed input.
bool parse_wkb(const uint8_t *data, size_t len, Geometry &out);

// Calls burn(col, row) for each grid cell the geometry covers, following
// GDALRasterizeGeometries' default (not all-touched) rules: the cell holding a
// point, one cell per step along the major axis of a line, the cells whose
// centre is inside a polygon (even-odd over all rings).
template <typename F>
void rasterize(const GeoReference &g, const Geometry &geom, F &&burn);

// Geo -> (col, row) through the inverse transform (crates/geometry/src/lib.rs:161-168).
inline void geo_to_pixel(const GeoReference &g, double x, double y, double &col, double &row) {
  const GT &v = g.transform.inv;
  col = (double)v.x0 + x * (double)v.dx + y * (double)v.rx;
  row = (double)v.y0 + x * (double)v.ry + y * (double)v.dy;
}

// Writes a single-band float32 GeoTIFF, tiled 256 x 256, with the geo
// transform and nodata = f32::MAX (crates/propag/src/propag.rs:576-600).
bool write_geotiff_f32(const std::string &path, const GeoReference &g, const float *data,
                       std::string &err);

// ---- template implementation -------------------------------------------------
template <typename F>
void rasterize(const GeoReference &g, const Geometry &geom, F &&burn) {
  const int64_t W = g.width, H = g.height;
  auto put = [&](int64_t c, int64_t r) {
    if (c >= 0 && r >= 0 && c < W && r < H) burn(c, r);
  };
  for (const Pt &p : geom.points) {
    double c, r;
    geo_to_pixel(g, p.x, p.y, c, r);
    put((int64_t)std::floor(c), (int64_t)std::floor(r));
  }
  for (const auto &line : geom.lines) {
    for (size_t k = 0; k + 1 < line.size(); ++k) {
      double c0, r0, c1, r1;
      geo_to_pixel(g, line[k].x, line[k].y, c0, r0);
      geo_to_pixel(g, line[k + 1].x, line[k + 1].y, c1, r1);
      const double dc = c1 - c0, dr = r1 - r0;
      const int64_t steps = (int64_t)std::ceil(std::max(std::fabs(dc), std::fabs(dr)));
      if (steps == 0) {
        put((int64_t)std::floor(c0), (int64_t)std::floor(r0));
        continue;
      }
      for (int64_t s = 0; s <= steps; ++s) {
        const double t = (double)s / (double)steps;
        put((int64_t)std::floor(c0 + t * dc), (int64_t)std::floor(r0 + t * dr));
      }
    }
  }
  for (const auto &poly : geom.polygons) {
    // pixel-space rings
    std::vector<std::vector<Pt>> rings;
    double rmin = 1e300, rmax = -1e300;
    for (const auto &ring : poly) {
      std::vector<Pt> pr;
      for (const Pt &p : ring) {
        Pt q;
        geo_to_pixel(g, p.x, p.y, q.x, q.y);
        rmin = std::min(rmin, q.y);
        rmax = std::max(rmax, q.y);
        pr.push_back(q);
      }
      rings.push_back(std::move(pr));
    }
    const int64_t r0 = std::max<int64_t>(0, (int64_t)std::floor(rmin));
    const int64_t r1 = std::min<int64_t>(H - 1, (int64_t)std::ceil(rmax));
    std::vector<double> xs;
    for (int64_t r = r0; r <= r1; ++r) {
      const double yc = (double)r + 0.5;
      xs.clear();
      for (const auto &ring : rings) {
        for (size_t k = 0; k + 1 < ring.size(); ++k) {
          const Pt a = ring[k], b = ring[k + 1];
          if ((a.y <= yc && b.y > yc) || (b.y <= yc && a.y > yc))
            xs.push_back(a.x + (yc - a.y) * (b.x - a.x) / (b.y - a.y));
        }
      }
      std::sort(xs.begin(), xs.end());
      for (size_t k = 0; k + 1 < xs.size(); k += 2) {
        // cells whose centre c + 0.5 lies in [xs[k], xs[k+1])
        const int64_t ca = (int64_t)std::ceil(xs[k] - 0.5);
        const int64_t cb = (int64_t)std::ceil(xs[k + 1] - 0.5) - 1;
        for (int64_t c = std::max<int64_t>(ca, 0); c <= std::min<int64_t>(cb, W - 1); ++c) put(c, r);
      }
    }
  }
}

}  // namespace propag
