/*
 * trk_constants.h -- physical and numerical constants shared by the device
 * kernels, the host element compiler and the CPU oracle.
 *
 * The reference takes c_mks, me_mev, e_mks, me_mks and PI from the SDDS
 * toolkit's constants.h / mdb.h, which the reference does not ship; it sets
 * particleMassMV = me_mev and particleRelSign = 1 for electrons
 * (src/elegant.c:2960-2967).  The values here are CODATA 2018 and IEEE double
 * pi; every consumer in this repository includes this one header, so the GPU
 * path, the oracle and the shim used to compile the reference sources agree
 * exactly.
 */
#ifndef TRK_CONSTANTS_H
#define TRK_CONSTANTS_H

#define TRK_C_MKS 2.99792458e8              /* speed of light, m/s (exact) */
#define TRK_ME_MEV 0.51099895000            /* electron rest energy, MeV */
#define TRK_E_MKS 1.602176634e-19           /* elementary charge, C (exact) */
#define TRK_ME_MKS 9.1093837015e-31         /* electron mass, kg */
#define TRK_RE_MKS 2.8179403262e-15         /* classical electron radius, m */
#define TRK_PI 3.141592653589793238462643
#define TRK_PIx2 6.283185307179586476925287
#define TRK_PIo2 1.570796326794896619231322
#define TRK_PARTICLE_REL_SIGN 1.0           /* electrons */
#define TRK_MU_O (4 * TRK_PI * 1e-7)        /* vacuum permeability, as the SDDS constants define it */
#define TRK_EPSILON_O (1 / (TRK_MU_O * TRK_C_MKS * TRK_C_MKS))

/* Loss limits on |x|,|y| and |x'|,|y'| inside kick elements (src/track.h:1250-1251,
 * global_settings.c:61-62 defaults). */
#define TRK_COORD_LIMIT 10.0
#define TRK_SLOPE_LIMIT 1.0

/* 2^(1/3), the Forest-Ruth coefficient (src/multipole.c:1086, src/csbend.c:1457) */
#define TRK_BETA 1.25992104989487316477

#endif
