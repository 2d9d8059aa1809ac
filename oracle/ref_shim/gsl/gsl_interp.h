#pragma once
#include "qshim_core.h"
