/*
 * thysea_dropin.h — the reference's own entry point, exported unchanged by
 * libthysea.so so that the reference's main() (src/ShallowWater.cxx) links
 * against this library instead of its CUDA code.
 *
 * Replaces: extern "C" int shallowWater(...)   src/GPU/ShallowWater.cu:182-190
 *           (declared by the caller at src/ShallowWater.cxx:19-27)
 *
 * The prototype is the reference's, including its C++ parameter types
 * (double2 and the tipoDatosSubmalla struct passed by value, std::string by
 * value), so it is link-compatible only with callers built with the same
 * C++ standard-library ABI.  Plain-C callers use thy_run / thy_run_netcdf in
 * thysea.h, which carry the same arguments in thy_problem.
 *
 * Behaviour kept: arguments are the dimensionless problem of
 * cargarDatosProblema(); outputs are <prefix>.nc when the NetCDF saving time
 * is >= 0 and <prefix>_ts.nc when gauges are read; *tiempo receives the
 * loop's wall time; returns 0, 1 (not enough GPU memory) or 2 (host memory
 * or NetCDF file error).  numNiveles must be 1.
 */
#ifndef THYSEA_DROPIN_H
#define THYSEA_DROPIN_H

#include <cstdint>
#include <string>
#include <vector_types.h>   /* double2 */

#ifndef THYSEA_NO_SUBMALLA_TYPE
/* layout of the reference's tipoDatosSubmalla (src/Constantes.hxx:32-38) */
using tipoDatosSubmalla = struct {
    double2 *areaYCosPhi;
    double *anchoVolumenes;
    double *altoVolumenes;
    double *longitud;
    double *latitud;
};
#endif

extern "C" int shallowWater(int numNiveles, int okada_flag, int numFaults, int crop_flag, double crop_value,
                            double *LON_C, double *LAT_C, double *DEPTH_C, double *FAULT_L, double *FAULT_W,
                            double *STRIKE, double *DIP, double *RAKE, double *SLIP, double *defTime,
                            double2 *datosVolumenesNivel_1, double2 *datosVolumenesNivel_2,
                            tipoDatosSubmalla datosNivel, int leer_fichero_puntos, int numPuntosGuardar,
                            int *posicionesVolumenesGuardado, double *lonPuntos, double *latPuntos,
                            int numVolxNivel0, int numVolyNivel0, int64_t numVolumenesNivel, double Hmin,
                            char *nombre_bati, std::string prefijo, double borde_sup, double borde_inf,
                            double borde_izq, double borde_der, int tam_spongeSup, int tam_spongeInf,
                            int tam_spongeIzq, int tam_spongeDer, double tiempo_tot, double tiempoGuardarNetCDF,
                            double tiempoGuardarSeries, double CFL, double mf0, double vmax, double epsilon_h,
                            double hpos, double cvis, double dif_at, double L, double H, double Q, double T,
                            char *version, double *tiempo);

#endif /* THYSEA_DROPIN_H */
