// Helper macros of FIR's public headers (src_lib/macros.h:1-48), same names
// and meaning, so that callers' loops over projection data compile unchanged.
#pragma once

#define ABS(a) ((a) < 0 ? (-(a)) : (a))
#define MIN(a, b) ((a) < (b) ? (a) : (b))
#define MAX(a, b) ((a) > (b) ? (a) : (b))

// Tolerance used by FIR's gates and Siddon tie rule
#define EPSILON 0.00001

#define PI 3.141592653589793

#define LOOP(INDEX, LO, HI) for (int INDEX = (LO); INDEX <= (HI); ++INDEX)

#define LOOP_SEG(SEG, PROJ) LOOP(SEG, -(PROJ).getGeometry().segOffset, (PROJ).getGeometry().segOffset)

#define LOOP_VIEW(VIEW, PROJ) LOOP(VIEW, 0, (PROJ).getGeometry().nViews - 1)

#define LOOP_AXIAL(AXIAL_COORD, PROJ, SEG) LOOP(AXIAL_COORD, 0, (PROJ).getGeometry().getNAxialCoords(SEG) - 1)

#define LOOP_TANG(TANG_COORD, PROJ)                                     \
  LOOP(TANG_COORD,                                                      \
       -(PROJ).getGeometry().tangCoordOffset,                           \
       -(PROJ).getGeometry().tangCoordOffset + (PROJ).getHeader().nTangCoords - 1)

// Bin of a segment by its index along the remaining dimensions
#define BIN(PROJ, SEG, BIN_INDEX) (PROJ).getDataArray()[(SEG) + (PROJ).getGeometry().segOffset][BIN_INDEX]
