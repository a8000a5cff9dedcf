// sparse_matrix.h — the umbrella header of the RVVLASparse API
// (include/sparse_matrix.h of the reference), for the GPU drop-in.
#pragma once

#include "CRS.h"
#include "CSR5.h"
#include "CVR.h"
#include "HCSR.h"
#include "LAV.h"
#include "SELL_C_Sigma.h"
#include "VHCC.h"
#include "VNEC.h"
#include "convert.h"
#include "spmv_mtx.h"
