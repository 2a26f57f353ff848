// Test infrastructure only (oracle build).  Declarations of the GSL random-number calls that the
// reference's src/particles.cpp makes in its random initial conditions and its sampler; the
// tree probe (oracle/tree_probe.cpp) calls neither, and its definitions of these functions
// abort if reached.
#pragma once
typedef struct gsl_rng_type gsl_rng_type;
typedef struct gsl_rng gsl_rng;
extern const gsl_rng_type* gsl_rng_taus;
gsl_rng* gsl_rng_alloc(const gsl_rng_type*);
void gsl_rng_set(const gsl_rng*, unsigned long int);
double gsl_rng_uniform(const gsl_rng*);
double gsl_rng_uniform_pos(const gsl_rng*);
unsigned long int gsl_rng_get(const gsl_rng*);
void gsl_rng_free(gsl_rng*);
