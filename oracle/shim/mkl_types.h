/* Test infrastructure (oracle): forwards to the MKL API stand-in. */
#pragma once
#include "mkl.h"
