/* See gflags.h in this directory: DECLARE_ forms only. */
#pragma once
#include "gflags.h"
