// engine_internal.h -- shared declarations of the engine's translation units.
#pragma once
#include <cstdarg>
#include <cstdint>

#include "../../include/smaug_b200.h"

namespace smaug {

// Thread-local last-error message; set_error returns `code` for chaining.
int set_error(int code, const char* fmt, ...);
void clear_error();
const char* last_error();

int grid_metric(int ndim, const int32_t* n, double* pos, double* delx);
int read_ini(const char* path, int ndim, const int32_t* n, double* w, double* pos, int32_t* it,
             double* t);
int write_out_host(const char* path, const smaug_params_t* p, const double* w, const double* pos,
                   const char* name, int32_t it, double t);

}  // namespace smaug
