#pragma once
// Qt header stand-in for the oracle/_ref harness (see qshim_core.h).
#include "qshim_core.h"
