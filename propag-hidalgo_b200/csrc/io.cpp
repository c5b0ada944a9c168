// WKB parsing and a minimal GeoTIFF writer (no GDAL in this build).
#include "io.hpp"

#include <cstdio>
#include <cstring>

namespace propag {
namespace {

struct Reader {
  const uint8_t *p;
  size_t n, at = 0;
  bool ok = true;
  bool need(size_t k) {
    if (!ok || at + k > n) ok = false;
    return ok;
  }
  uint32_t u32(bool le) {
    if (!need(4)) return 0;
    uint32_t v;
    if (le) {
      v = (uint32_t)p[at] | (uint32_t)p[at + 1] << 8 | (uint32_t)p[at + 2] << 16 |
          (uint32_t)p[at + 3] << 24;
    } else {
      v = (uint32_t)p[at + 3] | (uint32_t)p[at + 2] << 8 | (uint32_t)p[at + 1] << 16 |
          (uint32_t)p[at] << 24;
    }
    at += 4;
    return v;
  }
  double f64(bool le) {
    if (!need(8)) return 0;
    uint8_t b[8];
    for (int i = 0; i < 8; ++i) b[i] = le ? p[at + i] : p[at + 7 - i];
    at += 8;
    double v;
    std::memcpy(&v, b, 8);
    return v;
  }
};

bool parse_geom(Reader &r, Geometry &g, int depth) {
  if (depth > 8 || !r.need(1)) return false;
  const bool le = r.p[r.at++] == 1;
  uint32_t type = r.u32(le);
  bool has_z = false, has_m = false;
  if (type & 0x80000000u) has_z = true;  // EWKB flags
  if (type & 0x40000000u) has_m = true;
  if (type & 0x20000000u) r.u32(le);     // SRID
  type &= 0x0FFFFFFFu;
  if (type >= 3000) { has_z = has_m = true; type -= 3000; }
  else if (type >= 2000) { has_m = true; type -= 2000; }
  else if (type >= 1000) { has_z = true; type -= 1000; }
  const int extra = (has_z ? 1 : 0) + (has_m ? 1 : 0);
  auto point = [&](Pt &pt) {
    pt.x = r.f64(le);
    pt.y = r.f64(le);
    for (int e = 0; e < extra; ++e) r.f64(le);
    return r.ok;
  };
  auto seq = [&](std::vector<Pt> &out) {
    const uint32_t n = r.u32(le);
    if (!r.ok || n > r.n) return false;
    out.resize(n);
    for (uint32_t i = 0; i < n; ++i)
      if (!point(out[i])) return false;
    return true;
  };
  switch (type) {
    case 1: {
      Pt pt;
      if (!point(pt)) return false;
      if (!(std::isnan(pt.x) && std::isnan(pt.y))) g.points.push_back(pt);  // empty point
      return true;
    }
    case 2: {
      std::vector<Pt> line;
      if (!seq(line)) return false;
      g.lines.push_back(std::move(line));
      return true;
    }
    case 3: {
      const uint32_t nr = r.u32(le);
      if (!r.ok || nr > r.n) return false;
      std::vector<std::vector<Pt>> rings(nr);
      for (uint32_t i = 0; i < nr; ++i)
        if (!seq(rings[i])) return false;
      g.polygons.push_back(std::move(rings));
      return true;
    }
    case 4:
    case 5:
    case 6:
    case 7: {
      const uint32_t n = r.u32(le);
      if (!r.ok || n > r.n) return false;
      for (uint32_t i = 0; i < n; ++i)
        if (!parse_geom(r, g, depth + 1)) return false;
      return true;
    }
    default:
      return false;
  }
}

// ---- TIFF ------------------------------------------------------------------
struct TiffWriter {
  std::vector<uint8_t> buf;
  void u16(uint16_t v) { buf.push_back(v & 0xFF); buf.push_back(v >> 8); }
  void u32(uint32_t v) { for (int i = 0; i < 4; ++i) buf.push_back((v >> (8 * i)) & 0xFF); }
  void at32(size_t pos, uint32_t v) { for (int i = 0; i < 4; ++i) buf[pos + i] = (v >> (8 * i)) & 0xFF; }
};

}  // namespace

bool parse_wkb(const uint8_t *data, size_t len, Geometry &out) {
  if (!data || len < 5) return false;
  Reader r{data, len};
  Geometry g;
  if (!parse_geom(r, g, 0) || !r.ok) return false;
  out = std::move(g);
  return true;
}

void plan_geometry(const GeoReference &g, const Geometry &geom, int32_t feature, RasterPlan &plan) {
  const int64_t W = g.width, H = g.height;
  for (const Pt &p : geom.points) {
    double c, r;
    geo_to_pixel(g, p.x, p.y, c, r);
    plan_segment(plan, c, r, c, r, feature, W, H);
  }
  for (const auto &line : geom.lines)
    for (size_t k = 0; k + 1 < line.size(); ++k) {
      double c0, r0, c1, r1;
      geo_to_pixel(g, line[k].x, line[k].y, c0, r0);
      geo_to_pixel(g, line[k + 1].x, line[k + 1].y, c1, r1);
      plan_segment(plan, c0, r0, c1, r1, feature, W, H);
    }
  std::vector<std::vector<Pt>> rings;
  for (const auto &poly : geom.polygons) {
    rings.assign(poly.size(), {});
    for (size_t i = 0; i < poly.size(); ++i) {
      rings[i].resize(poly[i].size());
      for (size_t k = 0; k < poly[i].size(); ++k)
        geo_to_pixel(g, poly[i][k].x, poly[i][k].y, rings[i][k].x, rings[i][k].y);
    }
    plan_polygon(plan, rings, feature, H);
  }
}

bool write_geotiff_f32(const std::string &path, const GeoReference &g, const float *data,
                       std::string &err) {
  const uint32_t W = g.width, H = g.height, T = 256;
  const uint32_t tx = (W + T - 1) / T, ty = (H + T - 1) / T, nt = tx * ty;
  const std::string proj((const char *)g.proj, strnlen((const char *)g.proj, sizeof(g.proj)));
  const std::string nodata = "3.40282346638529e+38";
  const std::string citation = proj + "|";

  struct Entry {
    uint16_t tag, type;
    uint32_t count;
    std::vector<uint8_t> data;  // payload (little endian)
  };
  std::vector<Entry> e;
  auto add = [&](uint16_t tag, uint16_t type, uint32_t count, const void *p, size_t bytes) {
    Entry en{tag, type, count, std::vector<uint8_t>((const uint8_t *)p, (const uint8_t *)p + bytes)};
    e.push_back(std::move(en));
  };
  auto add_u16 = [&](uint16_t tag, uint16_t v) { add(tag, 3, 1, &v, 2); };
  auto add_u32 = [&](uint16_t tag, uint32_t v) { add(tag, 4, 1, &v, 4); };
  add_u32(256, W);
  add_u32(257, H);
  add_u16(258, 32);
  add_u16(259, 1);
  add_u16(262, 1);
  add_u16(277, 1);
  add_u16(284, 1);
  add_u16(322, (uint16_t)T);
  add_u16(323, (uint16_t)T);
  std::vector<uint32_t> offsets(nt, 0), counts(nt, T * T * 4);
  add(324, 4, nt, offsets.data(), nt * 4);  // patched below
  add(325, 4, nt, counts.data(), nt * 4);
  add_u16(339, 3);
  const GT &m = g.transform.gt;
  const double mt[16] = {m.dx, m.rx, 0, m.x0, m.ry, m.dy, 0, m.y0, 0, 0, 0, 0, 0, 0, 0, 1};
  add(34264, 12, 16, mt, sizeof(mt));  // ModelTransformationTag
  // GeoKeyDirectory: version 1.1.0, keys: GTRasterTypeGeoKey = PixelIsArea,
  // GTCitationGeoKey -> GeoAsciiParams (the PROJ string)
  const uint16_t keys[] = {1, 1, 0, 2, 1025, 0, 1, 1, 1026, 34737,
                           (uint16_t)citation.size(), 0};
  add(34735, 3, 12, keys, sizeof(keys));
  add(34737, 2, (uint32_t)citation.size() + 1, (citation + '\0').data(), citation.size() + 1);
  add(42113, 2, (uint32_t)nodata.size() + 1, (nodata + '\0').data(), nodata.size() + 1);

  TiffWriter w;
  w.buf.insert(w.buf.end(), {'I', 'I', 42, 0});
  w.u32(8);
  const size_t ifd = 8;
  const size_t ifd_size = 2 + e.size() * 12 + 4;
  size_t extra = ifd + ifd_size;
  // layout: IFD, then out-of-line payloads, then tiles
  w.buf.resize(extra, 0);
  std::vector<size_t> payload_at(e.size(), 0);
  for (size_t i = 0; i < e.size(); ++i) {
    if (e[i].data.size() > 4) {
      if (w.buf.size() & 1) w.buf.push_back(0);
      payload_at[i] = w.buf.size();
      w.buf.insert(w.buf.end(), e[i].data.begin(), e[i].data.end());
    }
  }
  while (w.buf.size() & 3) w.buf.push_back(0);
  const size_t tiles_at = w.buf.size();
  for (uint32_t t = 0; t < nt; ++t) offsets[t] = (uint32_t)(tiles_at + (size_t)t * T * T * 4);
  // the tile offsets: inline in the IFD entry when there is one tile (4 bytes),
  // else in the entry's out-of-line payload
  for (size_t i = 0; i < e.size(); ++i) {
    if (e[i].tag != 324) continue;
    std::memcpy(e[i].data.data(), offsets.data(), nt * 4);
    if (e[i].data.size() > 4) std::memcpy(w.buf.data() + payload_at[i], offsets.data(), nt * 4);
  }
  // IFD
  size_t at = ifd;
  auto put16 = [&](uint16_t v) { w.buf[at++] = v & 0xFF; w.buf[at++] = v >> 8; };
  auto put32 = [&](uint32_t v) { for (int i = 0; i < 4; ++i) w.buf[at++] = (v >> (8 * i)) & 0xFF; };
  put16((uint16_t)e.size());
  for (size_t i = 0; i < e.size(); ++i) {
    put16(e[i].tag);
    put16(e[i].type);
    put32(e[i].count);
    if (e[i].data.size() <= 4) {
      uint8_t v[4] = {0, 0, 0, 0};
      std::memcpy(v, e[i].data.data(), e[i].data.size());
      for (int k = 0; k < 4; ++k) w.buf[at++] = v[k];
    } else {
      put32((uint32_t)payload_at[i]);
    }
  }
  put32(0);
  // tiles (row-major tiles, padded with nodata)
  FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    err = "cannot open " + path;
    return false;
  }
  bool ok = std::fwrite(w.buf.data(), 1, w.buf.size(), f) == w.buf.size();
  std::vector<float> tile((size_t)T * T);
  for (uint32_t t = 0; t < nt && ok; ++t) {
    const uint32_t c0 = (t % tx) * T, r0 = (t / tx) * T;
    for (uint32_t r = 0; r < T; ++r)
      for (uint32_t c = 0; c < T; ++c) {
        const uint32_t gc = c0 + c, gr = r0 + r;
        tile[(size_t)r * T + c] = (gc < W && gr < H) ? data[(size_t)gr * W + gc] : 3.40282347e+38f;
      }
    ok = std::fwrite(tile.data(), 4, tile.size(), f) == tile.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) err = "write failed: " + path;
  return ok;
}

}  // namespace propag
