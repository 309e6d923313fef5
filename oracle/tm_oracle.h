// tm_oracle.h - CPU oracle of the reference's display transform,
// shaders/tonemapper-fragment-shader.glsl (TM:line), on the GLSL compat types.
//
// TEST INFRASTRUCTURE: compiled into the oracle library only (see pt_oracle.h).
#pragma once

namespace oracle {

struct ToneMapper {
  gfloat exposure, invGamma, contrast, saturation, hueShift;

  gfloat toneMap(gfloat L) { return L / (1.0f + L); }  // TM:14-17

  vec3 rgb2hsv(vec3 c) {  // TM:19-27
    vec4 K = vec4(0.0f, -1.0f / 3.0f, 2.0f / 3.0f, -1.0f);
    vec4 p = mix(vec4(c.b, c.g, K.w, K.z), vec4(c.g, c.b, K.x, K.y), step(c.b, c.g));
    vec4 q = mix(vec4(p.x, p.y, p.w, c.r), vec4(c.r, p.y, p.z, p.x), step(p.x, c.r));
    gfloat d = q.x - min(q.w, q.y);
    gfloat e = 1.0e-10f;
    return vec3(abs(q.z + (q.w - q.y) / (6.0f * d + e)), d / (q.x + e), q.x);
  }

  vec3 hsv2rgb(vec3 c) {  // TM:29-34
    vec4 K = vec4(1.0f, 2.0f / 3.0f, 1.0f / 3.0f, 3.0f);
    vec3 p = abs(fract(vec3(c.x) + vec3(K.x, K.y, K.z)) * 6.0f - vec3(K.w));
    return c.z * mix(vec3(K.x), clamp(p - vec3(K.x), 0.0f, 1.0f), c.y);
  }

  vec4 apply(vec3 L) {  // TM:36-97
    gfloat X = L.x, Y = L.y, Z = L.z;
    vec3 RGB;
    RGB.r = 3.2406f * X - 1.5372f * Y - 0.4986f * Z;
    RGB.g = -0.9689f * X + 1.8758f * Y + 0.0415f * Z;
    RGB.b = 0.0557f * X - 0.2040f * Y + 1.0570f * Z;
    gfloat delta = -min(gfloat(0.0f), min(min(RGB.r, RGB.g), RGB.b));
    RGB.r += delta;
    RGB.g += delta;
    RGB.b += delta;
    RGB = pow(RGB, vec3(invGamma));
    RGB *= pow(gfloat(2.0f), exposure);
    gfloat R = toneMap(RGB.r), G = toneMap(RGB.g), B = toneMap(RGB.b);
    gfloat mean = (R + G + B) / 3.0f;
    gfloat dR = R - mean, dG = G - mean, dB = B - mean;
    R = mean + sign(dR) * pow(abs(dR), 1.0f / saturation);
    G = mean + sign(dG) * pow(abs(dG), 1.0f / saturation);
    B = mean + sign(dB) * pow(abs(dB), 1.0f / saturation);
    dR = R - 0.5f;
    dG = G - 0.5f;
    dB = B - 0.5f;
    R = 0.5f + sign(dR) * pow(abs(dR), 1.0f / contrast);
    G = 0.5f + sign(dG) * pow(abs(dG), 1.0f / contrast);
    B = 0.5f + sign(dB) * pow(abs(dB), 1.0f / contrast);
    vec3 C = vec3(R, G, B);
    if (hueShift > 0.0f) {
      vec3 hsv = rgb2hsv(C);
      hsv.r = mod(hsv.r + hueShift, gfloat(1.0f));
      C = hsv2rgb(hsv);
    }
    return vec4(C.r, C.g, C.b, 1.0f);
  }
};

}  // namespace oracle
