// C restatements of the reference's live Fortran-77 kernels, for the oracle harness only
// (the container has no Fortran compiler).  Symbol names and argument order follow the
// Fortran calling convention the C++ sources declare in src/header/geoflow.h:153-179.
#include <cmath>

static double fsgn(double zz, double tiny) {  // src/geoflow/sgn.f:19-33
    double a = zz < 0. ? -zz : zz;
    if (a < tiny) return 0.0;
    if (zz >= tiny) return 1.0;
    return -1.0;
}

extern "C" {

// src/geoflow/getcoef.f:19-66
void gmfggetcoef_(double *uvec, double *dudx, double *dudy, double *dx, double *bedfrictang,
                  double *intfrictang, double *Kactx, double *Kacty, double *tiny, double *epsilon) {
    (void)dx;
    const double cosphi = std::cos(*intfrictang);
    const double tandel = std::tan(*bedfrictang);
    if (uvec[0] > *tiny) {
        const double vel = dudx[1] / uvec[0] - uvec[1] * dudx[0] / (uvec[0] * uvec[0]) + dudy[2] / uvec[0] -
                           uvec[2] * dudy[0] / (uvec[0] * uvec[0]);
        double ab = 1.0 - (1.0 + tandel * tandel) * (cosphi * cosphi);
        ab = ab < 0. ? -ab : ab;
        *Kactx = (2.0 / (cosphi * cosphi)) * (1.0 - fsgn(vel, *tiny) * std::sqrt(ab)) - 1.0;
        *Kacty = (2.0 / (cosphi * cosphi)) * (1.0 - fsgn(vel, *tiny) * std::sqrt(ab)) - 1.0;
        const double ux = uvec[1] / uvec[0], uy = uvec[2] / uvec[0];
        if ((ux < 0 ? -ux : ux) < *tiny && (uy < 0 ? -uy : uy) < *tiny) {
            *Kactx = 1.0;
            *Kacty = 1.0;
        }
        if (*Kactx < 0.0) {
            *Kactx = 0.0;
            *Kacty = 0.0;
        }
    } else {
        *Kactx = 1.0;
        *Kacty = 1.0;
    }
    *Kactx = *Kactx * *epsilon;
    *Kacty = *Kacty * *epsilon;
}

// src/geoflow/eigen.f:19-49
void eigen_(double *Uvec, double *eigenvxmax, double *eigenvymax, double *evalue, double *tiny, double *kactxy,
            double *gravity, double *v_solid, double *eps) {
    (void)eps;
    if (Uvec[0] > *tiny) {
        if (kactxy[0] < 0.0) {
            kactxy[0] = 0;
            kactxy[1] = 0;
        }
        *eigenvxmax = (v_solid[0] < 0 ? -v_solid[0] : v_solid[0]) + std::sqrt(kactxy[0] * gravity[2] * Uvec[0]);
        *eigenvymax = (v_solid[1] < 0 ? -v_solid[1] : v_solid[1]) + std::sqrt(kactxy[0] * gravity[2] * Uvec[0]);
    } else {
        *eigenvxmax = *tiny;
        *eigenvymax = *tiny;
    }
    *evalue = *eigenvxmax > *eigenvymax ? *eigenvxmax : *eigenvymax;
}

// src/geoflow/predict.f:19-45 has an empty body
void predict_(double *, double *, double *, double *, double *, double *, double *, double *, double *, double *,
              double *, double *, double *, int *, double *, int *, double *) {}
}
