// params.h -- parameter validation and the device parameter block, shared
// by the C-ABI translation units.
#ifndef LB3D_PARAMS_H
#define LB3D_PARAMS_H

#include <string>

#include "common.cuh"

namespace lb3d {

// Returns LB3DC_OK or an error code with the reason in `why`.
int validate_params(const lb3dc_params *p, std::string &why);
DevParams dev_params_from(const lb3dc_params &p);
// Records the message returned by lb3dc_last_error(NULL, ...).
int set_global_error(int code, const char *msg);

}  // namespace lb3d

#endif
