#pragma once
#include "gsl_rng.h"
