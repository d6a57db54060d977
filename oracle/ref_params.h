// ref_params.h -- TEST INFRASTRUCTURE.  The names of the reference's parameters.h at a chosen
// shape (PM_REF_W x PM_REF_H x PM_REF_D, default the reference's 640 x 480 x 64): defining that
// header's include guard first lets oracle/build_ref.py compile the reference's own sources,
// unmodified, at a small test shape.  The mutable parameters keep their definitions in the
// reference's parameters.cpp.  Included by ref_shim.h (CUDA sources) and ref_cpu_unity.cpp
// (the host-side CPU fusion variant).
#pragma once

#ifndef PM_REF_W
#define PM_REF_W 640
#endif
#ifndef PM_REF_H
#define PM_REF_H 480
#endif
#ifndef PM_REF_D
#define PM_REF_D 64
#endif

// ---- parameters.h at the test shape (same names the reference declares) ----------------
#define _parameters_h
#define FLOAT_EPS 1e-5
const int WIDTH = PM_REF_W;
const int HEIGHT = PM_REF_H;
extern int CASE;
const int DEP_CNT = PM_REF_D;
const float SAD_WEIGHT = 1.0f;
const int MARGIN = 2;
const int PATCH_SIZE = (2 * MARGIN + 1) * (2 * MARGIN + 1);
extern float pi1;
extern float pi2;
extern float tau_so;
extern float sgm_q1;
extern float sgm_q2;
extern float var_scale;
const float DEP_INF_1 = 2000.0f;
const float DEP_INF = 1000.0f;
const float COST_INF = 0.0f;

