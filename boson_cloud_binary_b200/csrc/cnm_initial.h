// cnm_initial.h -- host side of the device initial-state generators (cnm_initial.cu).
#pragma once

#include <string>

namespace cnm {

// The mode projection of the hydrogenic (n, la, ma) state of reduced mass mu about a body of
// mass M1 centred at x = x_center, normalised to sum |U|^2 dr = 1; state: interleaved complex,
// n_modes x Nr (host).  Returns a CNM_* status, with the message in err.
int hydrogenic_state(const double *r, int Nr, const int *l, const int *m, int n_modes, double mu, double M1,
                     double x_center, int n, int la, int ma, int n_theta, int n_phi, double *state, std::string &err);

}  // namespace cnm
