/*
 * Loads libpropag.so the way the reference's QGIS provider does
 * (qgis-plugin/propag-algo/src/plugincontainer.cpp:9-27: dlopen, then dlsym
 * of FFIPropagation_run and propag_rasterize_fuels) and runs one propagation
 * through a C terrain loader (qgis-plugin/propag-algo/src/qgspropagloader.h:
 * 26-41 fills the ten rasters).  Used by tests/test_qgis_harness.py.
 *
 *   qgis_harness <libpropag.so> <output.tif>
 * prints "ok" on success, else "error: <message>", and exits 0 either way
 * unless the library could not be loaded (exit 2).
 */
#include <dlfcn.h>
#include <stdio.h>
#include <string.h>

#include "propag_host.h"

static int calls = 0;

/* Uniform demo terrain (the reference's constant loader). */
static bool load(void *ctx, const GeoReference *g, FFITerrain *t) {
  (void)ctx;
  ++calls;
  const size_t n = (size_t)g->width * g->height;
  for (size_t i = 0; i < n; ++i) {
    t->fuel_code[i] = 1;
    t->d1hr[i] = t->d10hr[i] = t->d100hr[i] = t->herb[i] = t->wood[i] = 0.1f;
    t->wind_speed[i] = 5.0f;
    t->wind_azimuth[i] = 0.0f;
    t->slope[i] = 0.0f;
    t->aspect[i] = 0.0f;
  }
  return true;
}

int main(int argc, char **argv) {
  if (argc < 3) return 2;
  void *h = dlopen(argv[1], RTLD_LAZY);
  if (!h) {
    fprintf(stderr, "dlopen: %s\n", dlerror());
    return 2;
  }
  RunFn run = (RunFn)dlsym(h, "FFIPropagation_run");
  RasterizeFuelsFn fuels = (RasterizeFuelsFn)dlsym(h, "propag_rasterize_fuels");
  typedef bool (*SouthUp)(float, float, float, float, float, float, const char *, GeoReference *);
  SouthUp south_up = (SouthUp)dlsym(h, "GeoReference_south_up");
  if (!run || !fuels || !south_up) {
    fprintf(stderr, "dlsym failed\n");
    return 2;
  }
  const char *proj = "+proj=utm +zone=30 +ellps=GRS80 +units=m +no_defs";
  FFIPropagation p;
  memset(&p, 0, sizeof p);
  if (!south_up(0.0f, 0.0f, 640.0f, 640.0f, 5.0f, 5.0f, proj, &p.settings.geo_ref)) {
    printf("error: south_up\n");
    return 0;
  }
  p.settings.max_time = 3600.0f;
  /* one ignition point (little-endian WKB POINT) at the grid centre */
  unsigned char wkb[21] = {1, 1, 0, 0, 0};
  const double xy[2] = {322.5, 322.5};
  memcpy(wkb + 5, xy, 16);
  FFITimeFeature ign = {0.0f, wkb, sizeof wkb};
  p.output_path = argv[2];
  p.initial_ignited_elements = &ign;
  p.initial_ignited_elements_len = 1;
  p.initial_ignited_elements_crs = proj;
  p.terrain_loader.load = load;
  p.terrain_loader.context = NULL;
  char err[256];
  memset(err, 0, sizeof err);
  if (run(p, sizeof err - 1, err))
    printf("ok loads=%d\n", calls);
  else
    printf("error: %s\n", err);
  return 0;
}
