/*
 * rkf78_tableau.h -- Fehlberg's 7(8) Runge-Kutta pair as exact fractions.
 *
 * TEST INFRASTRUCTURE ONLY (shared by oracle_tdse.c and the odeint stand-in
 * under ref_shim/).  Source: E. Fehlberg, "Classical fifth-, sixth-, seventh-,
 * and eighth-order Runge-Kutta formulas with stepsize control", NASA TR R-287
 * (1968).  This is the method boost::odeint's runge_kutta_fehlberg78 applies
 * (used by the reference at src/tdse/tdse.cpp:171,190,254,273).  Each
 * coefficient becomes the double nearest p/q (p and q are exact doubles).
 */
#ifndef RKF78_TABLEAU_H_
#define RKF78_TABLEAU_H_

/* nodes c_s */
static const double RKF78_C[13][2] = {
    {0, 1}, {2, 27}, {1, 9}, {1, 6}, {5, 12}, {1, 2}, {5, 6},
    {1, 6}, {2, 3},  {1, 3}, {1, 1}, {0, 1},  {1, 1}};

/* non-zero a_{s,j} as (s, j, p, q) */
struct rkf78_entry { int s, j; double p, q; };
static const struct rkf78_entry RKF78_A[] = {
    {1, 0, 2, 27},
    {2, 0, 1, 36},       {2, 1, 1, 12},
    {3, 0, 1, 24},       {3, 2, 1, 8},
    {4, 0, 5, 12},       {4, 2, -25, 16},     {4, 3, 25, 16},
    {5, 0, 1, 20},       {5, 3, 1, 4},        {5, 4, 1, 5},
    {6, 0, -25, 108},    {6, 3, 125, 108},    {6, 4, -65, 27},
    {6, 5, 125, 54},
    {7, 0, 31, 300},     {7, 4, 61, 225},     {7, 5, -2, 9},
    {7, 6, 13, 900},
    {8, 0, 2, 1},        {8, 3, -53, 6},      {8, 4, 704, 45},
    {8, 5, -107, 9},     {8, 6, 67, 90},      {8, 7, 3, 1},
    {9, 0, -91, 108},    {9, 3, 23, 108},     {9, 4, -976, 135},
    {9, 5, 311, 54},     {9, 6, -19, 60},     {9, 7, 17, 6},
    {9, 8, -1, 12},
    {10, 0, 2383, 4100}, {10, 3, -341, 164},  {10, 4, 4496, 1025},
    {10, 5, -301, 82},   {10, 6, 2133, 4100}, {10, 7, 45, 82},
    {10, 8, 45, 164},    {10, 9, 18, 41},
    {11, 0, 3, 205},     {11, 5, -6, 41},     {11, 6, -3, 205},
    {11, 7, -3, 41},     {11, 8, 3, 41},      {11, 9, 6, 41},
    {12, 0, -1777, 4100},{12, 3, -341, 164},  {12, 4, 4496, 1025},
    {12, 5, -289, 82},   {12, 6, 2193, 4100}, {12, 7, 51, 82},
    {12, 8, 33, 164},    {12, 9, 12, 41},     {12, 11, 1, 1},
};
#define RKF78_NA ((int)(sizeof(RKF78_A) / sizeof(RKF78_A[0])))

/* 8th-order weights (the solution propagated) and 7th-order weights (used
 * only for the embedded error estimate) */
static const double RKF78_B8[13][2] = {
    {0, 1}, {0, 1}, {0, 1}, {0, 1}, {0, 1}, {34, 105}, {9, 35},
    {9, 35}, {9, 280}, {9, 280}, {0, 1}, {41, 840}, {41, 840}};
static const double RKF78_B7[13][2] = {
    {41, 840}, {0, 1}, {0, 1}, {0, 1}, {0, 1}, {34, 105}, {9, 35},
    {9, 35}, {9, 280}, {9, 280}, {41, 840}, {0, 1}, {0, 1}};

#endif
