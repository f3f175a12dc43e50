// Declarations of the libconfig calls milupHPC's material handler makes; the
// harness builds materials directly, so these stubs are never exercised.
// Test infrastructure only (oracle/ref_harness).
#pragma once
#define CONFIG_TRUE 1
#define CONFIG_FALSE 0
typedef struct config_setting_t { int unused; } config_setting_t;
typedef struct config_t { int unused; } config_t;
static inline void config_init(config_t*) {}
static inline void config_destroy(config_t*) {}
static inline int config_read_file(config_t*, const char*) { return CONFIG_FALSE; }
static inline const char* config_error_text(const config_t*) { return "libconfig unavailable"; }
static inline int config_error_line(const config_t*) { return 0; }
static inline config_setting_t* config_lookup(const config_t*, const char*) { return 0; }
static inline int config_setting_length(const config_setting_t*) { return 0; }
static inline config_setting_t* config_setting_get_elem(const config_setting_t*, unsigned int) { return 0; }
static inline config_setting_t* config_setting_get_member(const config_setting_t*, const char*) { return 0; }
static inline int config_setting_lookup_int(const config_setting_t*, const char*, int*) { return CONFIG_FALSE; }
static inline int config_setting_lookup_float(const config_setting_t*, const char*, double*) { return CONFIG_FALSE; }
