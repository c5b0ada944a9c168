// GeoPackage output of the reference's vector layers: the fire references
// (LineStrings from each burned cell's reference to the cell, layer
// "fire_references") and the outlines of the super-grid tiles ("grids") and
// of their thread blocks ("blocks"), as write_refs / write_boundaries write
// them through GDAL's GPKG driver (crates/propag/src/propag.rs:601-750).
//
// A GeoPackage is an SQLite database with a fixed set of metadata tables
// (OGC 12-128r18: gpkg_spatial_ref_sys, gpkg_contents,
// gpkg_geometry_columns) and one table per layer whose geometry column holds
// a GeoPackage binary header followed by the geometry in WKB.  SQLite is
// used through its C API from the system's runtime library
// (libsqlite3.so.0), loaded on first use; no GDAL.  The layer's CRS is the
// grid's projection string, which a GeoPackage wants as WKT: without a
// projection library the WKT is written for the CRSs whose definition needs
// no database (EPSG:4326, WGS 84 and ETRS89 UTM zones by EPSG code, PROJ
// strings of UTM or longitude/latitude on the WGS 84 or GRS 1980
// ellipsoid), and "undefined" for others; the srs row's description keeps
// the projection string either way.
#include <dlfcn.h>

#include <algorithm>
#include <cctype>
#include <cfloat>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "propag_b200.h"

namespace propag {
namespace {

// The SQLite C API entry points used here (public API, sqlite.org/c3ref).
struct Sqlite {
  void *lib = nullptr;
  int (*open_v2)(const char *, void **, int, const char *) = nullptr;
  int (*close)(void *) = nullptr;
  int (*exec)(void *, const char *, int (*)(void *, int, char **, char **), void *, char **) = nullptr;
  int (*prepare_v2)(void *, const char *, int, void **, const char **) = nullptr;
  int (*bind_blob)(void *, int, const void *, int, void (*)(void *)) = nullptr;
  int (*step)(void *) = nullptr;
  int (*reset)(void *) = nullptr;
  int (*finalize)(void *) = nullptr;
  const char *(*errmsg)(void *) = nullptr;
  void (*free_)(void *) = nullptr;
};
constexpr int kSqliteOk = 0, kSqliteDone = 101;
constexpr int kOpenReadWrite = 0x2, kOpenCreate = 0x4;

const Sqlite *sqlite(std::string &err) {
  static std::mutex mu;
  static Sqlite s;
  static bool tried = false;
  std::lock_guard<std::mutex> lk(mu);
  if (!tried) {
    tried = true;
    s.lib = dlopen("libsqlite3.so.0", RTLD_NOW | RTLD_LOCAL);
    if (s.lib) {
      auto sym = [&](const char *n) { return dlsym(s.lib, n); };
      s.open_v2 = (decltype(s.open_v2))sym("sqlite3_open_v2");
      s.close = (decltype(s.close))sym("sqlite3_close");
      s.exec = (decltype(s.exec))sym("sqlite3_exec");
      s.prepare_v2 = (decltype(s.prepare_v2))sym("sqlite3_prepare_v2");
      s.bind_blob = (decltype(s.bind_blob))sym("sqlite3_bind_blob");
      s.step = (decltype(s.step))sym("sqlite3_step");
      s.reset = (decltype(s.reset))sym("sqlite3_reset");
      s.finalize = (decltype(s.finalize))sym("sqlite3_finalize");
      s.errmsg = (decltype(s.errmsg))sym("sqlite3_errmsg");
      s.free_ = (decltype(s.free_))sym("sqlite3_free");
    }
  }
  if (!s.lib || !s.open_v2 || !s.close || !s.exec || !s.prepare_v2 || !s.bind_blob || !s.step ||
      !s.reset || !s.finalize || !s.errmsg || !s.free_) {
    err = "GeoPackage output needs SQLite's runtime library (libsqlite3.so.0)";
    return nullptr;
  }
  return &s;
}

// Little-endian appends.
void put_u32(std::vector<uint8_t> &b, uint32_t v) {
  for (int k = 0; k < 4; ++k) b.push_back((uint8_t)(v >> (8 * k)));
}
void put_f64(std::vector<uint8_t> &b, double v) {
  uint64_t u;
  std::memcpy(&u, &v, 8);
  for (int k = 0; k < 8; ++k) b.push_back((uint8_t)(u >> (8 * k)));
}

// A geometry as a GeoPackage blob: "GP", version 0, flags (little endian,
// envelope [minx, maxx, miny, maxy]), srs_id, envelope, then WKB
// (little endian; type 2 LineString or 3 Polygon with one ring).
std::vector<uint8_t> gpkg_blob(int32_t srs_id, bool polygon, const std::vector<double> &xy,
                               double env[4]) {
  std::vector<uint8_t> b = {'G', 'P', 0, 0x03};
  put_u32(b, (uint32_t)srs_id);
  env[0] = env[2] = DBL_MAX;
  env[1] = env[3] = -DBL_MAX;
  for (size_t i = 0; i + 1 < xy.size(); i += 2) {
    env[0] = std::min(env[0], xy[i]);
    env[1] = std::max(env[1], xy[i]);
    env[2] = std::min(env[2], xy[i + 1]);
    env[3] = std::max(env[3], xy[i + 1]);
  }
  for (int k = 0; k < 4; ++k) put_f64(b, env[k]);
  b.push_back(1);  // WKB little endian
  put_u32(b, polygon ? 3u : 2u);
  if (polygon) put_u32(b, 1u);  // one ring
  put_u32(b, (uint32_t)(xy.size() / 2));
  for (double v : xy) put_f64(b, v);
  return b;
}

std::string sql_quote(const std::string &s) {
  std::string o = "'";
  for (char c : s) {
    o += c;
    if (c == '\'') o += '\'';
  }
  return o + "'";
}

constexpr int32_t kCustomSrs = 100000;  // srs_id of a CRS without an EPSG code

// One row of gpkg_spatial_ref_sys for the grid's CRS.
struct SrsRow {
  int32_t id = kCustomSrs;
  std::string name = "grid", org = "NONE";
  int32_t org_id = kCustomSrs;
  std::string definition = "undefined", description;
};

// WKT 1 pieces (OGC 01-009) with the EPSG registry's names and constants.
const char *kWgs84Spheroid = "SPHEROID[\"WGS 84\",6378137,298.257223563,AUTHORITY[\"EPSG\",\"7030\"]]";
const char *kGrs80Spheroid = "SPHEROID[\"GRS 1980\",6378137,298.257222101,AUTHORITY[\"EPSG\",\"7019\"]]";
const char *kGreenwichDegree =
    "PRIMEM[\"Greenwich\",0,AUTHORITY[\"EPSG\",\"8901\"]],"
    "UNIT[\"degree\",0.0174532925199433,AUTHORITY[\"EPSG\",\"9122\"]]";

std::string wgs84_geogcs() {
  return std::string("GEOGCS[\"WGS 84\",DATUM[\"WGS_1984\",") + kWgs84Spheroid +
         ",AUTHORITY[\"EPSG\",\"6326\"]]," + kGreenwichDegree + ",AUTHORITY[\"EPSG\",\"4326\"]]";
}
std::string etrs89_geogcs() {
  return std::string("GEOGCS[\"ETRS89\",DATUM[\"European_Terrestrial_Reference_System_1989\",") +
         kGrs80Spheroid + ",TOWGS84[0,0,0,0,0,0,0],AUTHORITY[\"EPSG\",\"6258\"]]," + kGreenwichDegree +
         ",AUTHORITY[\"EPSG\",\"4258\"]]";
}
std::string unknown_geogcs(bool grs80) {
  return std::string("GEOGCS[\"unknown\",DATUM[\"Unknown based on ") + (grs80 ? "GRS 1980" : "WGS 84") +
         " ellipsoid\"," + (grs80 ? kGrs80Spheroid : kWgs84Spheroid) + "]," + kGreenwichDegree + "]";
}
// Universal Transverse Mercator zone 1-60 on `geogcs`; epsg = 0: no authority.
std::string utm_projcs(const std::string &name, const std::string &geogcs, int zone, bool south, int epsg) {
  std::string w = "PROJCS[\"" + name + "\"," + geogcs +
                  ",PROJECTION[\"Transverse_Mercator\"],PARAMETER[\"latitude_of_origin\",0],"
                  "PARAMETER[\"central_meridian\"," + std::to_string(6 * zone - 183) +
                  "],PARAMETER[\"scale_factor\",0.9996],PARAMETER[\"false_easting\",500000],"
                  "PARAMETER[\"false_northing\"," + (south ? "10000000" : "0") +
                  "],UNIT[\"metre\",1,AUTHORITY[\"EPSG\",\"9001\"]],AXIS[\"Easting\",EAST],"
                  "AXIS[\"Northing\",NORTH]";
  if (epsg) w += ",AUTHORITY[\"EPSG\",\"" + std::to_string(epsg) + "\"]";
  return w + "]";
}

bool parse_int(const std::string &s, int &v) {
  if (s.empty() || s.size() > 9) return false;
  v = 0;
  for (char c : s) {
    if (c < '0' || c > '9') return false;
    v = 10 * v + (c - '0');
  }
  return true;
}

SrsRow srs_row(const std::string &crs) {
  SrsRow r;
  r.description = crs;
  std::vector<std::string> tok;  // whitespace-separated words
  for (size_t i = 0; i < crs.size();) {
    while (i < crs.size() && std::isspace((unsigned char)crs[i])) ++i;
    size_t j = i;
    while (j < crs.size() && !std::isspace((unsigned char)crs[j])) ++j;
    if (j > i) tok.push_back(crs.substr(i, j - i));
    i = j;
  }
  auto lower = [](std::string t) {
    for (char &c : t) c = (char)std::tolower((unsigned char)c);
    return t;
  };
  int code = 0;
  if (tok.size() == 1 && lower(tok[0]).rfind("epsg:", 0) == 0 && parse_int(tok[0].substr(5), code)) {
    std::string def;
    if (code == 4326) def = wgs84_geogcs();
    else if ((code > 32600 && code <= 32660) || (code > 32700 && code <= 32760))
      def = utm_projcs("WGS 84 / UTM zone " + std::to_string(code % 100) + (code > 32700 ? "S" : "N"),
                       wgs84_geogcs(), code % 100, code > 32700, code);
    else if (code >= 25828 && code <= 25838)
      def = utm_projcs("ETRS89 / UTM zone " + std::to_string(code % 100) + "N", etrs89_geogcs(),
                       code % 100, false, code);
    if (def.empty()) return r;
    const size_t q = def.find('"') + 1;
    r.id = r.org_id = code;
    r.org = "EPSG";
    r.name = def.substr(q, def.find('"', q) - q);
    r.definition = def;
    return r;
  }
  // a PROJ string: +proj=utm|longlat|latlong, +zone, +south, +ellps / +datum,
  // +units=m; anything else leaves the CRS undefined
  std::string proj, ellps;
  int zone = 0;
  bool south = false;
  for (const std::string &t : tok) {
    if (t.size() < 2 || t[0] != '+') return r;
    const size_t eq = t.find('=');
    const std::string key = t.substr(1, eq == std::string::npos ? std::string::npos : eq - 1);
    const std::string val = eq == std::string::npos ? "" : t.substr(eq + 1);
    if (key == "proj") proj = val;
    else if (key == "zone") {
      if (!parse_int(val, zone)) return r;
    } else if (key == "south" && val.empty()) south = true;
    else if (key == "ellps" || key == "datum") {
      if (val != "WGS84" && val != "GRS80") return r;
      if (!ellps.empty() && ellps != val) return r;
      ellps = val;
    } else if (key == "units") {
      if (val != "m") return r;
    } else if (key == "towgs84") {
      if (val != "0,0,0" && val != "0,0,0,0,0,0,0") return r;
    } else if (key != "no_defs" && !(key == "type" && val == "crs")) {
      return r;
    }
  }
  if (ellps.empty()) return r;
  const bool grs80 = ellps == "GRS80";
  if (proj == "utm" && zone >= 1 && zone <= 60)
    r.definition = utm_projcs("unknown", grs80 ? unknown_geogcs(true) : wgs84_geogcs(), zone, south, 0);
  else if ((proj == "longlat" || proj == "latlong") && zone == 0 && !south)
    r.definition = grs80 ? unknown_geogcs(true) : wgs84_geogcs();
  if (r.definition != "undefined") r.name = "unknown";
  return r;
}

// Writes one layer (a new file at `path`) with one feature per geometry
// (flat x, y pairs); geom_type "LINESTRING" or "POLYGON".
bool write_layer(const std::string &path, const char *layer, bool polygon,
                 const std::vector<std::vector<double>> &geoms, const std::string &crs,
                 std::string &err) {
  const Sqlite *s = sqlite(err);
  if (!s) return false;
  std::remove(path.c_str());  // a new GeoPackage, as GDAL's create does
  void *db = nullptr;
  if (s->open_v2(path.c_str(), &db, kOpenReadWrite | kOpenCreate, nullptr) != kSqliteOk) {
    err = "cannot create GeoPackage " + path + (db ? std::string(": ") + s->errmsg(db) : "");
    if (db) s->close(db);
    return false;
  }
  auto exec = [&](const std::string &sql) {
    char *msg = nullptr;
    if (s->exec(db, sql.c_str(), nullptr, nullptr, &msg) != kSqliteOk) {
      err = "GeoPackage " + path + ": " + (msg ? msg : "SQL error");
      if (msg) s->free_(msg);
      return false;
    }
    return true;
  };
  const std::string t = layer, gt = polygon ? "POLYGON" : "LINESTRING";
  const SrsRow srs = srs_row(crs);
  double ext[4] = {DBL_MAX, -DBL_MAX, DBL_MAX, -DBL_MAX};
  bool ok =
      exec("PRAGMA application_id = 1196444487; PRAGMA user_version = 10200; BEGIN;") &&
      exec("CREATE TABLE gpkg_spatial_ref_sys (srs_name TEXT NOT NULL, srs_id INTEGER NOT NULL "
           "PRIMARY KEY, organization TEXT NOT NULL, organization_coordsys_id INTEGER NOT NULL, "
           "definition TEXT NOT NULL, description TEXT);") &&
      exec("INSERT INTO gpkg_spatial_ref_sys VALUES ('Undefined cartesian SRS', -1, 'NONE', -1, "
           "'undefined', 'undefined cartesian coordinate reference system'), "
           "('Undefined geographic SRS', 0, 'NONE', 0, 'undefined', "
           "'undefined geographic coordinate reference system'), "
           "('WGS 84 geodetic', 4326, 'EPSG', 4326, 'GEOGCS[\"WGS 84\",DATUM[\"WGS_1984\","
           "SPHEROID[\"WGS 84\",6378137,298.257223563,AUTHORITY[\"EPSG\",\"7030\"]],"
           "AUTHORITY[\"EPSG\",\"6326\"]],PRIMEM[\"Greenwich\",0,AUTHORITY[\"EPSG\",\"8901\"]],"
           "UNIT[\"degree\",0.0174532925199433,AUTHORITY[\"EPSG\",\"9122\"]],"
           "AUTHORITY[\"EPSG\",\"4326\"]]', 'longitude/latitude coordinates in decimal degrees "
           "on the WGS 84 spheroid');") &&
      (srs.id == 4326 ||
       exec("INSERT INTO gpkg_spatial_ref_sys VALUES (" + sql_quote(srs.name) + ", " +
            std::to_string(srs.id) + ", " + sql_quote(srs.org) + ", " + std::to_string(srs.org_id) + ", " +
            sql_quote(srs.definition) + ", " + sql_quote(srs.description) + ");")) &&
      exec("CREATE TABLE gpkg_contents (table_name TEXT NOT NULL PRIMARY KEY, data_type TEXT NOT "
           "NULL, identifier TEXT UNIQUE, description TEXT DEFAULT '', last_change DATETIME NOT "
           "NULL DEFAULT (strftime('%Y-%m-%dT%H:%M:%fZ','now')), min_x DOUBLE, min_y DOUBLE, "
           "max_x DOUBLE, max_y DOUBLE, srs_id INTEGER, CONSTRAINT fk_gc_r_srs_id FOREIGN KEY "
           "(srs_id) REFERENCES gpkg_spatial_ref_sys(srs_id));") &&
      exec("CREATE TABLE gpkg_geometry_columns (table_name TEXT NOT NULL, column_name TEXT NOT "
           "NULL, geometry_type_name TEXT NOT NULL, srs_id INTEGER NOT NULL, z TINYINT NOT NULL, "
           "m TINYINT NOT NULL, CONSTRAINT pk_geom_cols PRIMARY KEY (table_name, column_name), "
           "CONSTRAINT fk_gc_tn FOREIGN KEY (table_name) REFERENCES gpkg_contents(table_name), "
           "CONSTRAINT fk_gc_srs FOREIGN KEY (srs_id) REFERENCES gpkg_spatial_ref_sys (srs_id));") &&
      exec("CREATE TABLE \"" + t + "\" (fid INTEGER PRIMARY KEY AUTOINCREMENT NOT NULL, geom " + gt +
           ");");
  if (ok) {
    void *st = nullptr;
    const std::string ins = "INSERT INTO \"" + t + "\" (geom) VALUES (?);";
    ok = s->prepare_v2(db, ins.c_str(), -1, &st, nullptr) == kSqliteOk;
    for (size_t i = 0; ok && i < geoms.size(); ++i) {
      double env[4];
      const std::vector<uint8_t> blob = gpkg_blob(srs.id, polygon, geoms[i], env);
      ext[0] = std::min(ext[0], env[0]);
      ext[1] = std::max(ext[1], env[1]);
      ext[2] = std::min(ext[2], env[2]);
      ext[3] = std::max(ext[3], env[3]);
      ok = s->bind_blob(st, 1, blob.data(), (int)blob.size(), (void (*)(void *))-1) == kSqliteOk &&
           s->step(st) == kSqliteDone && s->reset(st) == kSqliteOk;
    }
    if (!ok) err = "GeoPackage " + path + ": " + s->errmsg(db);
    if (st) s->finalize(st);
  }
  if (ok) {
    char b[256];
    if (geoms.empty()) ext[0] = ext[1] = ext[2] = ext[3] = 0.0;
    std::snprintf(b, sizeof(b), "%.17g, %.17g, %.17g, %.17g", ext[0], ext[2], ext[1], ext[3]);
    ok = exec("INSERT INTO gpkg_contents (table_name, data_type, identifier, min_x, min_y, max_x, "
              "max_y, srs_id) VALUES (" + sql_quote(t) + ", 'features', " + sql_quote(t) + ", " + b +
              ", " + std::to_string(srs.id) + ");") &&
         exec("INSERT INTO gpkg_geometry_columns VALUES (" + sql_quote(t) + ", 'geom', '" + gt +
              "', " + std::to_string(srs.id) + ", 0, 0);") &&
         exec("COMMIT;");
  }
  s->close(db);
  return ok;
}

// Cell corner (c, r) of the grid in world coordinates (GeoReference::backward).
void world(const GeoReference &g, double c, double r, std::vector<double> &xy) {
  const GT &t = g.transform.gt;
  xy.push_back((double)t.x0 + c * (double)t.dx + r * (double)t.rx);
  xy.push_back((double)t.y0 + c * (double)t.ry + r * (double)t.dy);
}

std::string crs_of(const GeoReference &g) {
  return std::string((const char *)g.proj, strnlen((const char *)g.proj, sizeof(g.proj)));
}

}  // namespace

bool write_refs_gpkg(const GeoReference &g, const float *time, const uint16_t *rx,
                     const uint16_t *ry, const std::string &path, std::string &err) {
  // the reference's loop order: columns outer, rows inner (propag.rs:713-716)
  std::vector<std::vector<double>> geoms;
  for (uint32_t i = 0; i < g.width; ++i)
    for (uint32_t j = 0; j < g.height; ++j) {
      const uint64_t ix = i + (uint64_t)j * g.width;
      if (!(time[ix] < FLT_MAX)) continue;
      std::vector<double> xy;
      world(g, rx[ix] + 0.5, ry[ix] + 0.5, xy);  // from the reference's cell centre
      world(g, i + 0.5, j + 0.5, xy);            // to the cell's centre
      geoms.push_back(std::move(xy));
    }
  return write_layer(path, "fire_references", false, geoms, crs_of(g), err);
}

bool write_boundaries_gpkg(const GeoReference &g, uint32_t tile, uint32_t block,
                           const std::string &grid_path, const std::string &block_path,
                           std::string &err) {
  const uint32_t sx = (g.width + tile - 1) / tile, sy = (g.height + tile - 1) / tile;
  std::vector<std::vector<double>> grids, blocks;
  auto rect = [&](double c0, double r0, double c1, double r1) {
    std::vector<double> xy;
    world(g, c0, r0, xy);
    world(g, c1, r0, xy);
    world(g, c1, r1, xy);
    world(g, c0, r1, xy);
    world(g, c0, r0, xy);
    return xy;
  };
  for (uint32_t gy = 0; gy < sy; ++gy)
    for (uint32_t gx = 0; gx < sx; ++gx) {
      grids.push_back(rect(gx * tile, gy * tile, (gx + 1) * tile, (gy + 1) * tile));
      for (uint32_t by = 0; by < tile / block; ++by)
        for (uint32_t bx = 0; bx < tile / block; ++bx)
          blocks.push_back(rect(gx * tile + bx * block, gy * tile + by * block,
                                gx * tile + (bx + 1) * block, gy * tile + (by + 1) * block));
    }
  const std::string crs = crs_of(g);
  if (!grid_path.empty() && !write_layer(grid_path, "grids", true, grids, crs, err)) return false;
  if (!block_path.empty() && !write_layer(block_path, "blocks", true, blocks, crs, err)) return false;
  return true;
}

}  // namespace propag
