// Internal helpers shared by the library's translation units (not part of the ABI).
#pragma once
#include <stdint.h>

#include "../../include/p2r.h"

// Records `msg` as the calling thread's last error and returns `code`.
int p2r_set_error(int code, const char* msg);
// printf-style variant.
int p2r_set_errorf(int code, const char* fmt, ...);
// Clears the calling thread's last error; returns P2R_OK.
int p2r_clear_error();

// Validates the sizes of a p2r_config; returns P2R_OK or P2R_ERR_INVALID with a message.
int p2r_check_config(const p2r_config* cfg, const char* who);

// kfact exactly as the reference rounds it (TBB:654); bz == 0 means 3.8112 T.
float p2r_kfact_of(double bz);
