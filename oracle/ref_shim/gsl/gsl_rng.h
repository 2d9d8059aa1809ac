#pragma once
// gsl_rng stand-in: the type only (the generator is never used on the path)
typedef struct gsl_rng gsl_rng;
