/* Declaration of the one MKL PARDISO entry the reference solver calls
 * (solver/MG/Elasticity_Matrix.cpp:211,225,253,278), for building the
 * reference with oracle/ref_solver/ref_support.cpp instead of MKL.  Test
 * infrastructure only. */
#pragma once
extern "C" void pardiso_64(void* pt, const long long* maxfct, const long long* mnum, const long long* mtype,
                           const long long* phase, const long long* n, const void* a, const long long* ia,
                           const long long* ja, long long* perm, const long long* nrhs, long long* iparm,
                           const long long* msglvl, void* b, void* x, long long* error);
