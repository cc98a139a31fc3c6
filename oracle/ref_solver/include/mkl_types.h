/* Stand-in for MKL's type header, which the reference includes but whose
 * names it does not use (solver/MG/Elasticity_Matrix.cpp:10).  Test
 * infrastructure only. */
#pragma once
