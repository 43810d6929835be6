/* Minimal build configuration used only to compile STIR's
   RayTraceVoxelsOnCartesianGrid.cxx from the STIR tree into oracle/_ref
   (little-endian x86-64, no optional libraries, TOF-enabled headers). */
#ifndef __stir_config__H__
#define __stir_config__H__
#define STIR_VERSION 060500
#define STIR_VERSION_STRING "6.5.0"
#define LITTLE_ENDIAN_BYTE_ORDER_FROM_CMAKE
#define USE_PMRT
#define STIR_TOF 1
#endif
