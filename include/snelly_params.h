// snelly_params.h - the per-job parameter block of the spectral path tracer.
//
// One field per uniform the reference host uploads before drawing a frame
// (js/renderer.js:520-584 camera/settings/lights, js/materials.js:72-83 Surface,
// :245-275 Volume, :497-501 Metal, :752-762 Dielectric), already converted the way the
// host converts them (10^x powers, lengthScale products). Shared verbatim by the host
// runtime (C++), the CUDA kernels (NVRTC) and the CPU oracle, so it is plain C: floats,
// ints and fixed arrays, 4-byte aligned apart from the trailing pointers.
#pragma once

#define SNELLY_PARAMS_VERSION 1

// Dielectric IOR models (js/materials.js:833-1099).
#define SNELLY_IOR_ABBE 0        // coeffs: iorVal, abbe
#define SNELLY_IOR_SELLMEIER 1   // n^2 = 1 + C1 + sum C2t l^2 / (l^2 - C2t+1^2)
#define SNELLY_IOR_SELLMEIER2 2  // n^2 = 1 + C1 + sum C2t l^2 / (l^2 - C2t+1)
#define SNELLY_IOR_POLYANSKIY 3  // n^2 = C1 + C2 l^C3 / (l^2 - C4^C5)
#define SNELLY_IOR_CAUCHY 4      // n = C1 + sum C2t l^C2t+1
#define SNELLY_MAX_IOR_COEFFS 16
#define SNELLY_METAL_SAMPLES 64  // n,k samples over 390..750 nm (js/materials.js:536-627)
#define SNELLY_XYZ_SAMPLES 1024  // CIE XYZ table texels (js/color.js:24-284)
#define SNELLY_ICDF_SAMPLES 4096 // emission inverse-CDF texels (js/spectra.js:28-61)

typedef struct SnellyParams {
  // image / camera (js/renderer.js:520-536)
  float resolution[2];
  float camPos[3], camDir[3], camX[3], camY[3];
  float camFovy, camAspect, camAperture, camFocalDistance;
  // path-tracing settings (js/renderer.js:547-559)
  float filterRadius, radianceClamp, skipProbability, shadowStrength;
  int maxStepsIsMiss, wavelengthSamples, maxSSSSteps;
  int maxBounces;  // per-job bound on path vertices, <= the module's MAX_BOUNCES (0: the module's)
  float lengthScale, minLengthScale, maxLengthScale, pad1;
  // sky (js/renderer.js:562-569)
  int haveEnvMap, envMapVisible;
  float envMapPhiRotation, envMapThetaRotation, envMapTransitionAngle, skyPower;
  float skyTintUp[3], skyTintDown[3];
  // sun (js/renderer.js:570-578, updateSunDir :371-383)
  float sunPower, sunAngularSize, sunLatitude, sunLongitude;
  float sunColor[3], sunDir[3];
  int sunVisibleDirectly, pad2;
  // sphere light (js/renderer.js:580-583)
  float sphereLightPosition[3], sphereLightRadius, sphereLightPower, sphereLightColor[3];
  // metal (js/materials.js:497-501)
  float metalRoughness, metalSpecAlbedoRGB[3];
  // dielectric (js/materials.js:752-762)
  float dieleRoughness, dieleAbsorptionRGB[3], dieleSpecAlbedoRGB[3];
  // surface (js/materials.js:72-83)
  float surfaceDiffuseAlbedoRGB[3], surfaceSpecAlbedoRGB[3], surfaceRoughness, surfaceIor;
  float subsurface, subsurfaceAlbedoRGB[3], subsurfaceMFP, subsurfaceAnisotropy, subsurfaceDiffuseWeight;
  // atmosphere + fog + volumetric emission (js/materials.js:245-275)
  float atmosphereBoundsMin[3], atmosphereBoundsMax[3];
  float atmosphereExtinctionCoeffRGB[3], atmosphereScatteringCoeffRGB[3];
  float atmosphereMFP, atmosphereAnisotropy;
  int fogEnable;
  float fogMaxOpticalDepth, fogMFP, fogEmission[3], fogTint[3];
  float volumeEmission, volumeEmissionColorRGB[3];
  // dielectric IOR model and its coefficients (js/materials.js:1125-1147)
  int dieleModel, dieleNumCoeffs;
  float dieleCoeffs[SNELLY_MAX_IOR_COEFFS];
  // metal n and k, 64 samples each over 390..750 nm
  float metalN[SNELLY_METAL_SAMPLES], metalK[SNELLY_METAL_SAMPLES];
  // device pointers (set by the runtime): XYZ table (1024 x 4 floats), emission ICDF
  // (4096 floats), optional lat-long environment map (sRGB8, RGB, envMapW x envMapH).
  const float* xyzTable;
  const float* icdfTable;
  const unsigned char* envMap;
  int envMapW, envMapH;
} SnellyParams;
