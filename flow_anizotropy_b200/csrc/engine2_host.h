// D2Q9 host helpers shared by the 2D entry points (not part of the ABI).
#pragma once
#include "../../include/lbm.h"
#include "engine2d.cuh"

struct lbm_ctx;

// Parameter checks: tau > 0.5, and the positive lag / sample of LMB2d/main.cpp:304.
int check_params2d(lbm_ctx *ctx, const lbm_params2d &p);
// Solve record of one direction (everything but the device pointers).
void fill_solve2(lbm::Solve2 &S, int nx, int ny, const double F[2], const lbm_params2d &p);
// Controller state at step 0.
void init_state2(lbm::State2 &st, const lbm::Ctl2 &c);
