/*
 * rt_spectral_tables.h — measured spectral data shared by the renderer and its
 * CPU checker.  These are published data sets, not code; both sides must hold
 * the same numbers, so they live in one header.
 *
 *  - CIE 1931 2° standard observer colour-matching functions, 5 nm steps,
 *    380–700 nm (65 samples) — the range the reference tabulates
 *    (src/spectrum.rs:7-62).
 *  - Johnson & Christy (1972) complex refractive index (n, k) of gold, copper
 *    and silver, 25 nm steps from 380 nm (13 samples), as tabulated by the
 *    reference (src/spectrum.rs:213-225).
 *
 * Plain C, usable from host C/C++ and CUDA device code alike (the CUDA side
 * copies them into __constant__ memory).
 */
#ifndef RT_SPECTRAL_TABLES_H
#define RT_SPECTRAL_TABLES_H

#define RT_CIE_N      65
#define RT_CIE_START  380.0f
#define RT_CIE_STEP   5.0f

/* x̄(λ), ȳ(λ), z̄(λ) interleaved per wavelength: {x, y, z} at 380, 385, … 700 nm */
static const float RT_CIE_XYZ[RT_CIE_N][3] = {
    {0.001368f, 0.000039f, 0.006450f}, {0.002236f, 0.000064f, 0.010550f},
    {0.004243f, 0.000120f, 0.020050f}, {0.007650f, 0.000217f, 0.036210f},
    {0.014310f, 0.000396f, 0.067850f}, {0.023190f, 0.000640f, 0.110200f},
    {0.043510f, 0.001210f, 0.207400f}, {0.077630f, 0.002180f, 0.371300f},
    {0.134380f, 0.004000f, 0.645600f}, {0.214770f, 0.007300f, 1.039050f},
    {0.283900f, 0.011600f, 1.385600f}, {0.328500f, 0.016840f, 1.622960f},
    {0.348280f, 0.023000f, 1.747060f}, {0.348060f, 0.029800f, 1.782600f},
    {0.336200f, 0.038000f, 1.772110f}, {0.318700f, 0.048000f, 1.744100f},
    {0.290800f, 0.060000f, 1.669200f}, {0.251100f, 0.073900f, 1.528100f},
    {0.195360f, 0.090980f, 1.287640f}, {0.142100f, 0.112600f, 1.041900f},
    {0.095640f, 0.139020f, 0.812950f}, {0.057950f, 0.169300f, 0.616200f},
    {0.032010f, 0.208020f, 0.465180f}, {0.014700f, 0.258600f, 0.353300f},
    {0.004900f, 0.323000f, 0.272000f}, {0.002400f, 0.407300f, 0.212300f},
    {0.009300f, 0.503000f, 0.158200f}, {0.029100f, 0.608200f, 0.111700f},
    {0.063270f, 0.710000f, 0.078250f}, {0.109600f, 0.793200f, 0.057250f},
    {0.165500f, 0.862000f, 0.042160f}, {0.225750f, 0.914850f, 0.029840f},
    {0.290400f, 0.954000f, 0.020300f}, {0.359700f, 0.980300f, 0.013400f},
    {0.433450f, 0.994950f, 0.008750f}, {0.512050f, 1.000000f, 0.005750f},
    {0.594500f, 0.995000f, 0.003900f}, {0.678400f, 0.978600f, 0.002750f},
    {0.762100f, 0.952000f, 0.002100f}, {0.842500f, 0.915400f, 0.001800f},
    {0.916300f, 0.870000f, 0.001650f}, {0.978600f, 0.816300f, 0.001400f},
    {1.026300f, 0.757000f, 0.001100f}, {1.056700f, 0.694900f, 0.001000f},
    {1.062200f, 0.631000f, 0.000800f}, {1.045600f, 0.566800f, 0.000600f},
    {1.002600f, 0.503000f, 0.000340f}, {0.938400f, 0.441200f, 0.000240f},
    {0.854450f, 0.381000f, 0.000190f}, {0.751400f, 0.321000f, 0.000100f},
    {0.642400f, 0.265000f, 0.000050f}, {0.541900f, 0.217000f, 0.000030f},
    {0.447900f, 0.175000f, 0.000020f}, {0.360800f, 0.138200f, 0.000010f},
    {0.283500f, 0.107000f, 0.000000f}, {0.218700f, 0.081600f, 0.000000f},
    {0.164900f, 0.061000f, 0.000000f}, {0.121200f, 0.044580f, 0.000000f},
    {0.087400f, 0.032000f, 0.000000f}, {0.063600f, 0.023200f, 0.000000f},
    {0.046770f, 0.017000f, 0.000000f}, {0.032900f, 0.011920f, 0.000000f},
    {0.022700f, 0.008210f, 0.000000f}, {0.015840f, 0.005723f, 0.000000f},
    {0.011359f, 0.004102f, 0.000000f},
};

/* Extension of the table past 700 nm (705–780 nm, 16 samples) for the
 * 380–780 nm sampling range.  The reference stops at 700 nm and clamps beyond
 * it.  These values are the Wyman–Sloan–Shirley (JCGT 2013) multi-lobe
 * Gaussian fit of the 1931 CMFs, scaled per channel so that the fit meets the
 * tabulated 700 nm value:
 *   ext(λ) = table(700) · fit(λ) / fit(700)
 *   x̄ fit: 1.056 g(599.8, 37.9, 31.0) + 0.362 g(442.0, 16.0, 26.7) − 0.065 g(501.1, 20.4, 26.2)
 *   ȳ fit: 0.821 g(568.8, 46.9, 40.5) + 0.286 g(530.9, 16.3, 31.1)
 *   z̄ fit: 0   (the tabulated z̄ is already 0 from 650 nm)
 *   g(μ, σ1, σ2) = exp(−½((λ−μ)/σ)²), σ = σ1 below μ and σ2 above. */
#define RT_CIE_EXT_N 16
static const float RT_CIE_XYZ_EXT[RT_CIE_EXT_N][3] = {
    {6.657015e-03f, 2.728918e-03f, 0.0f}, {3.801202e-03f, 1.788000e-03f, 0.0f},
    {2.114776e-03f, 1.153789e-03f, 0.0f}, {1.146331e-03f, 7.332740e-04f, 0.0f},
    {6.054208e-04f, 4.589732e-04f, 0.0f}, {3.115350e-04f, 2.829367e-04f, 0.0f},
    {1.561919e-04f, 1.717798e-04f, 0.0f}, {7.629779e-05f, 1.027154e-04f, 0.0f},
    {3.631345e-05f, 6.048950e-05f, 0.0f}, {1.683934e-05f, 3.508366e-05f, 0.0f},
    {7.608248e-06f, 2.004059e-05f, 0.0f}, {3.349240e-06f, 1.127449e-05f, 0.0f},
    {1.436514e-06f, 6.246891e-06f, 0.0f}, {6.003099e-07f, 3.408879e-06f, 0.0f},
    {2.444236e-07f, 1.832061e-06f, 0.0f}, {9.696451e-08f, 9.697258e-07f, 0.0f},
};

#define RT_METAL_NK_N      13
#define RT_METAL_NK_START  380.0f
#define RT_METAL_NK_STEP   25.0f

/* [metal][0 = n, 1 = k][sample] for gold, copper, silver */
static const float RT_METAL_NK[3][2][RT_METAL_NK_N] = {
    { /* gold */
        {1.69f, 1.65f, 1.54f, 1.33f, 0.97f, 0.54f, 0.30f, 0.23f, 0.20f, 0.19f, 0.18f, 0.16f, 0.16f},
        {1.91f, 1.94f, 1.95f, 1.92f, 1.80f, 1.93f, 2.41f, 3.00f, 3.56f, 4.07f, 4.56f, 4.99f, 5.41f},
    },
    { /* copper */
        {1.23f, 1.21f, 1.16f, 1.10f, 1.04f, 0.88f, 0.60f, 0.38f, 0.26f, 0.22f, 0.21f, 0.20f, 0.21f},
        {2.00f, 2.26f, 2.49f, 2.59f, 2.64f, 2.69f, 2.84f, 3.21f, 3.70f, 4.17f, 4.64f, 5.07f, 5.48f},
    },
    { /* silver */
        {0.18f, 0.14f, 0.12f, 0.13f, 0.13f, 0.13f, 0.14f, 0.14f, 0.15f, 0.16f, 0.16f, 0.17f, 0.17f},
        {1.57f, 2.01f, 2.50f, 3.02f, 3.55f, 4.05f, 4.54f, 5.02f, 5.50f, 5.98f, 6.42f, 6.84f, 7.22f},
    },
};

#endif /* RT_SPECTRAL_TABLES_H */
