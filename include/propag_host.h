/*
 * propag_host.h -- the extern "C" plugin ABI of libpropag.so.
 *
 * These are the names and repr(C) layouts that the reference's host crate
 * exports (its cbindgen-generated `propag_host.h` / `geometry.h`, see
 * crates/propag/build.rs:20-44, which the reference does not ship) and that
 * its QGIS provider binds with dlopen/dlsym
 * (qgis-plugin/propag-algo/src/plugincontainer.cpp:9-27).  A host written
 * against the reference library links or dlopens this one unchanged.
 *
 * Each declaration cites the reference item it replaces (paths relative to
 * the reference project).
 */
#ifndef PROPAG_HOST_H
#define PROPAG_HOST_H

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Halo of a propagation block, in cells.  crates/propag/src/propag.rs:31
 * (a pub const, which cbindgen emits into the reference's header) */
#define HALO_RADIUS 1

/* Affine geo transform (GDAL order).  crates/geometry/src/lib.rs:20-28 */
typedef struct GT {
  float x0;
  float dx;
  float rx;
  float y0;
  float ry;
  float dy;
} GT;

/* Transform and its inverse.  crates/geometry/src/lib.rs:127-131 */
typedef struct GeoTransform {
  GT gt;
  GT inv;
} GeoTransform;

/* Grid size, projection and transform.  crates/geometry/src/lib.rs:180-187 */
typedef struct GeoReference {
  uint32_t width;
  uint32_t height;
  uint8_t proj[1024];
  GeoTransform transform;
} GeoReference;

/* crates/propag/src/propag.rs:38-43 */
typedef struct Settings {
  GeoReference geo_ref;
  float max_time;
} Settings;

/* Per-cell fire used by the propagation.  crates/propag/src/propag.rs:53-60 */
typedef struct FireSimpleCuda {
  float speed_max;    /* m/s */
  float azimuth_max;  /* rad */
  float eccentricity; /* - */
} FireSimpleCuda;

/* An ignition: a WKB geometry in `initial_ignited_elements_crs` burning at
 * `time` seconds.  crates/propag/src/propag.rs:120-125 */
typedef struct FFITimeFeature {
  float time;
  const uint8_t *geom_wkb;
  uintptr_t geom_wkb_len;
} FFITimeFeature;

/* A fuel polygon for propag_rasterize_fuels.  crates/propag/src/propag.rs:150-155 */
typedef struct FFIFuelFeature {
  uint8_t code;
  const uint8_t *geom_wkb;
  uintptr_t geom_wkb_len;
} FFIFuelFeature;

/* Callee-owned terrain rasters (width*height each) that a LoadFn fills.
 * crates/propag/src/propag.rs:763-775 */
typedef struct FFITerrain {
  uint8_t *fuel_code;
  float *d1hr;
  float *d10hr;
  float *d100hr;
  float *herb;
  float *wood;
  float *wind_speed;   /* m/s */
  float *wind_azimuth; /* rad, bearing the wind blows toward */
  float *slope;        /* rise / run */
  float *aspect;       /* rad, downslope azimuth */
} FFITerrain;

/* crates/propag/src/propag.rs:783 */
typedef bool (*LoadFn)(void *context, const GeoReference *geo_ref, FFITerrain *terrain);

/* crates/propag/src/propag.rs:777-781 */
typedef struct FFITerrainLoader {
  LoadFn load;
  void *context;
} FFITerrainLoader;

/* crates/propag/src/propag.rs:177-188 */
typedef struct FFIPropagation {
  Settings settings;
  const char *output_path;
  const char *refs_output_path;
  const char *block_boundaries_out_path;
  const char *grid_boundaries_out_path;
  const FFITimeFeature *initial_ignited_elements;
  uintptr_t initial_ignited_elements_len;
  const char *initial_ignited_elements_crs;
  FFITerrainLoader terrain_loader;
} FFIPropagation;

/* crates/propag/src/propag.rs:784-794 */
typedef bool (*RunFn)(FFIPropagation propag, uintptr_t err_len, char *err_msg);
typedef bool (*RasterizeFuelsFn)(const FFIFuelFeature *fuels, uintptr_t fuels_len,
                                 const char *fuels_crs, const GeoReference *geo_ref,
                                 uint8_t *result, char *err_msg, uintptr_t err_len);

/* crates/propag/src/propag.rs:796-801 */
typedef struct PluginT {
  RunFn run;
  RasterizeFuelsFn rasterize_fuels;
} PluginT;

/* Runs fire behaviour + propagation on the GPU and writes the arrival-time
 * GeoTIFF to output_path (refs / boundary outputs: see the file writers).
 * Returns false and strncpy()s a message into err_msg on error.  Unlike the
 * reference it may be called any number of times per process.
 * Replaces FFIPropagation_run, crates/propag/src/propag.rs:272-309. */
bool FFIPropagation_run(FFIPropagation propag, uintptr_t err_len, char *err_msg);

/* Burns fuel codes of WKB polygons into result (width*height bytes,
 * nodata 255).  Replaces propag_rasterize_fuels,
 * crates/propag/src/propag.rs:892-927 (GDAL-free: geometries must already be
 * in the grid's CRS). */
bool propag_rasterize_fuels(const FFIFuelFeature *fuels, uintptr_t fuels_len,
                            const char *fuels_crs, const GeoReference *geo_ref, uint8_t *result,
                            char *err_msg, uintptr_t err_len);

/* crates/propag/src/propag.rs:802-811 */
PluginT create_plugin(void);

/* crates/propag/src/propag.rs:45-51 */
Settings create_settings(GeoReference geo_ref, float max_time);

/* crates/propag/src/propag.rs:62-81 */
FireSimpleCuda create_fire(float speed_max, float azimuth_max, float eccentricity);

/* crates/geometry/src/lib.rs:195-238 */
uint32_t GeoReference_len(const GeoReference *self);
float GeoReference_x0(const GeoReference *self);
float GeoReference_x1(const GeoReference *self);
float GeoReference_y0(const GeoReference *self);
float GeoReference_y1(const GeoReference *self);

/* crates/geometry/src/lib.rs:277-332 */
bool GeoReference_south_up(float x0, float y0, float x1, float y1, float dx, float dy,
                           const char *proj, GeoReference *result);
bool GeoReference_north_up(float x0, float y0, float x1, float y1, float dx, float dy,
                           const char *proj, GeoReference *result);

#ifdef __cplusplus
}
#endif

#endif /* PROPAG_HOST_H */
