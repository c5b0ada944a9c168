// GDAL-free geometry and raster I/O used by the plugin ABI.
#pragma once

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "propag_host.h"
#include "raster.hpp"

namespace propag {

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
// GDALRasterizeGeometries' default (not all-touched) rules (raster.hpp): the
// cell holding a point, one cell per step along the major axis of a line, the
// cells whose centre is inside a polygon (even-odd over all rings).
template <typename F>
void rasterize(const GeoReference &g, const Geometry &geom, F &&burn);

// Appends the geometry of feature `feature` to a plan, in pixel space.
void plan_geometry(const GeoReference &g, const Geometry &geom, int32_t feature, RasterPlan &plan);

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
  RasterPlan plan;
  plan_geometry(g, geom, 0, plan);
  run_plan_host(plan, g.width, g.height, [&](int32_t, int64_t c, int64_t r) { burn(c, r); });
}

}  // namespace propag
