/*
 * constants.h - the reference's compile-time constants and enums
 * (src/constants.h:1-14), with the same names and values, since callers of
 * dtfe.h index tetra_data and tri_data rows with them.
 */
#ifndef SDTFE_CONSTANTS_H
#define SDTFE_CONSTANTS_H

#include <float.h>

#define ZERO (1e4 * DBL_EPSILON) /* |Plücker product| below this counts as 0 */
#define DIM 3
#define PERTURB_MAX 1000

typedef enum { BDC, ACD, ADB, ABC } face_t;         /* face k is opposite vertex k */
typedef enum { CB, AC, BA, DC, BD, DA } side_t;     /* tet edges                   */
typedef enum { A, B, C, D } vertex_t;

#endif
