/* The reference includes fftw3.h globally (Definitions.cpp:76) but its hot path
 * never calls FFTW.  Only the planner flag it reads is provided. */
#pragma once
#define FFTW_ESTIMATE 0
