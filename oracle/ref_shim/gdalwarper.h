/* Test infrastructure: see gdal_priv.h in this folder. */
#pragma once
#include "gdal_priv.h"
