/*
 * Symplectic integrators selectable by the GPU tracking call's ``integrator``
 * argument (the reference GPU backend's gpupass: atgpu/PyInterface.cpp:44-50,
 * coefficients atgpu/SymplecticIntegrator.cpp:28-80).  One integration step
 * of length SL = Length/NumIntSteps is, for i = 0..n-1, a drift of SL*c[i]
 * followed by a kick of SL*d[i], a zero coefficient skipping its drift or
 * kick.  The values equal the reference backend's to the last bit (tracking
 * results depend on them; tests/golden/integrators.json pins them):
 *   1  Euler, one drift and one kick
 *   2  McLachlan & Atela's optimal second-order method (Nonlinearity 5, 1992)
 *   3  Ruth's third-order method (IEEE Trans. Nucl. Sci. 30, 1983)
 *   4  Forest & Ruth's fourth-order method, the CPU engine's (Physica D 43, 1990)
 *   5  McLachlan & Atela's optimal fourth-order method
 *   6  Yoshida's sixth-order method, solution A (Phys. Lett. A 150, 1990)
 * Entry 0 is unused: tables compiled for the default integrator keep their
 * Forest-Ruth drift and kick lengths in the element record instead.
 */
#ifndef ATB_INTEGRATORS_H
#define ATB_INTEGRATORS_H

#define ATB_INTEG_MAX_STAGES 8
#define ATB_INTEG_COUNT 7

struct AtbInteg {
    int n;
    double c[ATB_INTEG_MAX_STAGES];
    double d[ATB_INTEG_MAX_STAGES];
};

static __constant__ AtbInteg atb_integ[ATB_INTEG_COUNT] = {
    {0, {0.0}, {0.0}},
    {1, {1.0}, {1.0}},
    {2, {0.29289321881345254, 0.7071067811865475},
        {0.29289321881345254, 0.7071067811865475}},
    {3, {1.0, -0.6666666666666666, 0.6666666666666666},
        {-0.041666666666666664, 0.75, 0.2916666666666667}},
    {4, {0.6756035959798289, -0.17560359597982889, -0.17560359597982889, 0.6756035959798289},
        {1.3512071919596578, -1.7024143839193155, 1.3512071919596578, 0.0}},
    {4, {0.1288461583653843, 0.4415830236164665, -0.0857820194129737, 0.5153528374311229},
        {0.3340036032863214, 0.7563200005156683, -0.2248198030794208, 0.1344961992774311}},
    {8, {0.39225680523878, 0.5100434119184585, -0.4710533854097566, 0.0687531682525181,
         0.0687531682525181, -0.4710533854097566, 0.5100434119184585, 0.39225680523878},
        {0.78451361047756, 0.235573213359357, -1.17767998417887, 1.3151863206839063,
         -1.17767998417887, 0.235573213359357, 0.78451361047756, 0.0}},
};

#endif  // ATB_INTEGRATORS_H
