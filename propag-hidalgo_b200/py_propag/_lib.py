"""ctypes binding of libpropag.so (include/propag_host.h, include/propag_b200.h).

The structures below mirror the C declarations field for field.  Loading
fails loudly when the library has not been built: there is no Python or CPU
implementation of the hot path behind this module.
"""
from __future__ import annotations

import ctypes as C
import os

PKG_DIR = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(PKG_DIR, "libpropag.so")

PROPAG_OK = 0
PROPAG_ERR_INVALID = -1
PROPAG_ERR_CUDA = -2
PROPAG_ERR_NO_DEVICE = -3
PROPAG_ERR_TIMEOUT = -4
PROPAG_ERR_OOM = -5
PROPAG_DEFAULT_TILE = 323
PROPAG_TILE_WHOLE_GRID = -1
PROPAG_CLUSTER_GROUPS = -1  # PropagOptions.cluster: teams of CTAs over the whole device
PROPAG_ARITH_REFERENCE = 0  # time_from with the reference's operations (CUDA atan2f, __cosf, contracted)
PROPAG_ARITH_PORTABLE = 1   # time_from with portable operations a CPU reproduces bit for bit


class GT(C.Structure):
    _fields_ = [("x0", C.c_float), ("dx", C.c_float), ("rx", C.c_float),
                ("y0", C.c_float), ("ry", C.c_float), ("dy", C.c_float)]


class GeoTransform(C.Structure):
    _fields_ = [("gt", GT), ("inv", GT)]


class GeoReference(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("proj", C.c_uint8 * 1024),
                ("transform", GeoTransform)]


class Settings(C.Structure):
    _fields_ = [("geo_ref", GeoReference), ("max_time", C.c_float)]


class FireSimpleCuda(C.Structure):
    _fields_ = [("speed_max", C.c_float), ("azimuth_max", C.c_float), ("eccentricity", C.c_float)]


class FFITimeFeature(C.Structure):
    _fields_ = [("time", C.c_float), ("geom_wkb", C.POINTER(C.c_uint8)), ("geom_wkb_len", C.c_size_t)]


class FFIFuelFeature(C.Structure):
    _fields_ = [("code", C.c_uint8), ("geom_wkb", C.POINTER(C.c_uint8)), ("geom_wkb_len", C.c_size_t)]


class FFITerrain(C.Structure):
    _fields_ = [("fuel_code", C.POINTER(C.c_uint8))] + [
        (k, C.POINTER(C.c_float)) for k in ("d1hr", "d10hr", "d100hr", "herb", "wood", "wind_speed",
                                            "wind_azimuth", "slope", "aspect")]


LoadFn = C.CFUNCTYPE(C.c_bool, C.c_void_p, C.POINTER(GeoReference), C.POINTER(FFITerrain))


class FFITerrainLoader(C.Structure):
    _fields_ = [("load", LoadFn), ("context", C.c_void_p)]


class FFIPropagation(C.Structure):
    _fields_ = [("settings", Settings), ("output_path", C.c_char_p), ("refs_output_path", C.c_char_p),
                ("block_boundaries_out_path", C.c_char_p), ("grid_boundaries_out_path", C.c_char_p),
                ("initial_ignited_elements", C.POINTER(FFITimeFeature)),
                ("initial_ignited_elements_len", C.c_size_t),
                ("initial_ignited_elements_crs", C.c_char_p), ("terrain_loader", FFITerrainLoader)]


RunFn = C.CFUNCTYPE(C.c_bool, FFIPropagation, C.c_size_t, C.c_char_p)
RasterizeFuelsFn = C.CFUNCTYPE(C.c_bool, C.POINTER(FFIFuelFeature), C.c_size_t, C.c_char_p,
                               C.POINTER(GeoReference), C.POINTER(C.c_uint8), C.c_char_p, C.c_size_t)


class PluginT(C.Structure):
    _fields_ = [("run", RunFn), ("rasterize_fuels", RasterizeFuelsFn)]


TERRAIN_FIELDS = ("fuel_code", "d1hr", "d10hr", "d100hr", "herb", "wood", "wind_speed",
                  "wind_azimuth", "slope", "aspect")


class PropagTerrainPtrs(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in TERRAIN_FIELDS]


FIRE_FIELDS = ("rx_int", "speed0", "hpua", "phi_eff_wind", "speed_max", "azimuth_max",
               "eccentricity", "residence_time", "byrams_max", "flame_max")


class PropagFireFields(C.Structure):
    _fields_ = [(k, C.c_void_p) for k in FIRE_FIELDS]


class PropagIgnition(C.Structure):
    _fields_ = [("x", C.c_uint32), ("y", C.c_uint32), ("time", C.c_float)]


class PropagOptions(C.Structure):
    _fields_ = [("tile", C.c_int32), ("cluster", C.c_int32), ("threads", C.c_int32), ("device", C.c_int32),
                ("arith", C.c_int32)]


PROPAG_STATIC_MAX_CELLS = 1 << 20  # propag_run_device_static's fixed scratch

STAT_FIELDS = ("rounds", "launches", "sweeps", "evaluations", "improvements", "dda_steps",
               "refbox_scans", "burned", "gathers", "cyc_first", "cyc_eval", "cyc_commit",
               "cyc_stage")


class PropagStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in STAT_FIELDS] + [("status", C.c_uint32),
                                                         ("max_walk", C.c_uint32),
                                                         ("t_start_ns", C.c_uint64),
                                                         ("t_done_ns", C.c_uint64),
                                                         ("scan_cells", C.c_uint64),
                                                         ("cyc_wait", C.c_uint64)]

    def as_dict(self):
        return {k: int(getattr(self, k)) for k in STAT_FIELDS + ("status", "max_walk", "t_start_ns", "t_done_ns",
                                                                   "scan_cells", "cyc_wait")}


class PropagJob(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("dx", C.c_float), ("dy", C.c_float),
                ("max_time", C.c_float), ("tile", C.c_int32),
                ("speed_max", C.c_void_p), ("azimuth_max", C.c_void_p), ("eccentricity", C.c_void_p),
                ("ignitions", C.c_void_p), ("n_ignitions", C.c_uint32), ("arith", C.c_uint32),
                ("time", C.c_void_p), ("refs_x", C.c_void_p), ("refs_y", C.c_void_p),
                ("boundaries", C.c_void_p)]


class PropagWeatherPtrs(C.Structure):
    _fields_ = [("temperature", C.c_void_p), ("humidity", C.c_void_p), ("cloud_cover", C.c_void_p),
                ("precipitation", C.c_void_p)]


class PropagServerOptions(C.Structure):
    _fields_ = [("hbm_budget", C.c_uint64), ("lanes", C.c_uint32), ("max_batch", C.c_uint32),
                ("device", C.c_int32), ("pad", C.c_int32)]


class PropagServerResult(C.Structure):
    _fields_ = [("stats", PropagStats), ("submit_ns", C.c_uint64), ("start_ns", C.c_uint64),
                ("done_ns", C.c_uint64), ("status", C.c_int32), ("batch_size", C.c_uint32),
                ("message", C.c_char * 128)]


# name -> (restype, argtypes); every symbol of both headers
SIGNATURES = {
    "FFIPropagation_run": (C.c_bool, [FFIPropagation, C.c_size_t, C.c_char_p]),
    "propag_rasterize_fuels": (C.c_bool, [C.POINTER(FFIFuelFeature), C.c_size_t, C.c_char_p,
                                          C.POINTER(GeoReference), C.c_void_p, C.c_char_p, C.c_size_t]),
    "create_plugin": (PluginT, []),
    "create_settings": (Settings, [GeoReference, C.c_float]),
    "create_fire": (FireSimpleCuda, [C.c_float, C.c_float, C.c_float]),
    "GeoReference_len": (C.c_uint32, [C.POINTER(GeoReference)]),
    "GeoReference_x0": (C.c_float, [C.POINTER(GeoReference)]),
    "GeoReference_x1": (C.c_float, [C.POINTER(GeoReference)]),
    "GeoReference_y0": (C.c_float, [C.POINTER(GeoReference)]),
    "GeoReference_y1": (C.c_float, [C.POINTER(GeoReference)]),
    "GeoReference_south_up": (C.c_bool, [C.c_float] * 6 + [C.c_char_p, C.POINTER(GeoReference)]),
    "GeoReference_north_up": (C.c_bool, [C.c_float] * 6 + [C.c_char_p, C.POINTER(GeoReference)]),
    "propag_last_error": (C.c_char_p, []),
    "propag_device_count": (C.c_int, []),
    "propag_version": (C.c_char_p, []),
    "propag_fire_simple_device": (C.c_int, [C.c_uint64, C.POINTER(PropagTerrainPtrs), C.c_void_p,
                                            C.c_void_p, C.c_void_p, C.c_void_p]),
    "propag_fire_full_device": (C.c_int, [C.c_uint64, C.POINTER(PropagTerrainPtrs),
                                          C.POINTER(PropagFireFields), C.c_void_p]),
    "propag_fire_simple_host": (C.c_int, [C.c_uint64, C.POINTER(PropagTerrainPtrs), C.c_void_p,
                                          C.c_void_p, C.c_void_p]),
    "propag_fire_full_host": (C.c_int, [C.c_uint64, C.POINTER(PropagTerrainPtrs),
                                        C.POINTER(PropagFireFields)]),
    "propag_engine_create": (C.c_void_p, [C.POINTER(PropagOptions)]),
    "propag_engine_job_bytes": (C.c_uint64, [C.c_uint32, C.c_uint32]),
    "propag_engine_destroy": (None, [C.c_void_p]),
    "propag_engine_run": (C.c_int, [C.c_void_p, C.POINTER(PropagJob), C.c_uint32, C.c_void_p,
                                    C.POINTER(PropagStats)]),
    "propag_engine_last_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_float * 3)]),
    "propag_selftest_group_wait": (C.c_int, [C.POINTER(C.c_uint32)]),
    "propag_selftest_time_from": (C.c_int, [C.c_int, C.c_uint64] + [C.c_void_p] * 8 +
                                  [C.c_float, C.c_float, C.c_void_p]),
    "propag_selftest_cosf_table": (C.c_int, [C.c_uint32, C.c_uint64, C.c_void_p]),
    "propag_selftest_atan2f_table": (C.c_int, [C.c_int32, C.c_int32, C.c_void_p]),
    "propag_slope_aspect_device": (C.c_int, [C.c_uint32, C.c_uint32, C.c_double, C.c_double, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p]),
    "propag_dmoist_device": (C.c_int, [C.c_uint64, C.c_int, C.c_int, C.POINTER(PropagWeatherPtrs),
                                       C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p,
                                       C.c_void_p, C.c_void_p, C.c_void_p]),
    "propag_fire_weather_device": (C.c_int, [C.c_uint64, C.c_int, C.c_int, C.POINTER(PropagWeatherPtrs),
                                             C.POINTER(PropagTerrainPtrs), C.c_void_p, C.c_void_p,
                                             C.c_void_p, C.c_void_p]),
    "propag_dmoist_host": (C.c_int, [C.c_uint64, C.c_int, C.c_int, C.POINTER(PropagWeatherPtrs),
                                     C.c_void_p, C.c_void_p, C.c_void_p, C.c_float, C.c_void_p,
                                     C.c_void_p, C.c_void_p]),
    "propag_engine_last_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PropagStats), C.c_uint32]),
    "propag_server_create": (C.c_void_p, [C.POINTER(PropagServerOptions)]),
    "propag_server_submit": (C.c_int64, [C.c_void_p, C.POINTER(PropagJob), C.POINTER(PropagTerrainPtrs),
                                         C.c_uint64]),
    "propag_server_poll": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(PropagServerResult)]),
    "propag_server_wait": (C.c_int, [C.c_void_p, C.c_int64, C.POINTER(PropagServerResult), C.c_uint32]),
    "propag_server_release": (C.c_int, [C.c_void_p, C.c_int64]),
    "propag_server_destroy": (None, [C.c_void_p]),
    "propag_graph_create": (C.c_void_p, [C.POINTER(PropagOptions), C.POINTER(PropagJob),
                                         C.POINTER(PropagTerrainPtrs), C.c_uint32]),
    "propag_graph_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "propag_graph_stats": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(PropagStats)]),
    "propag_graph_destroy": (None, [C.c_void_p]),
    "propag_autotune": (C.c_int, [C.POINTER(PropagJob), C.POINTER(PropagTerrainPtrs), C.c_uint32,
                                  C.c_void_p, C.c_int, C.POINTER(PropagOptions),
                                  C.POINTER(C.c_float)]),
    "propag_run_device_static": (C.c_int, [C.POINTER(PropagJob), C.c_void_p, C.POINTER(PropagStats)]),
    "propag_static_last_status": (C.c_int, [C.c_void_p, C.POINTER(PropagStats)]),
    "propag_run_host": (C.c_int, [C.POINTER(Settings), C.POINTER(PropagTerrainPtrs),
                                  C.POINTER(PropagIgnition), C.c_uint64, C.POINTER(PropagOptions),
                                  C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.POINTER(PropagStats)]),
    "propag_rasterize_ignitions": (C.c_int64, [C.POINTER(GeoReference), C.POINTER(FFITimeFeature),
                                               C.c_uint64, C.POINTER(PropagIgnition), C.c_uint64]),
    "propag_rasterize_times_device": (C.c_int, [C.POINTER(GeoReference), C.POINTER(FFITimeFeature),
                                                C.c_uint64, C.c_void_p, C.c_void_p]),
    "propag_rasterize_fuels_device": (C.c_int, [C.POINTER(FFIFuelFeature), C.c_size_t, C.c_char_p,
                                                C.POINTER(GeoReference), C.c_void_p, C.c_void_p]),
    "propag_ignitions_from_times_device": (C.c_int64, [C.c_void_p, C.c_uint32, C.c_uint32, C.c_void_p,
                                                       C.c_uint64, C.c_void_p]),
    "propag_write_geotiff": (C.c_int, [C.POINTER(GeoReference), C.c_void_p, C.c_char_p]),
    "propag_write_refs_gpkg": (C.c_int, [C.POINTER(GeoReference), C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_char_p]),
    "propag_write_boundaries_gpkg": (C.c_int, [C.POINTER(GeoReference), C.c_int32, C.c_char_p,
                                               C.c_char_p]),
}

_lib = None


class LibraryMissing(ImportError):
    pass


def lib():
    """The loaded libpropag.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                f"{LIB_PATH} is not built; run `make -C propag-hidalgo_b200/csrc` "
                "(there is no CPU fallback)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def last_error() -> str:
    msg = lib().propag_last_error()
    return msg.decode() if msg else ""
