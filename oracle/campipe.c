/* C restatement of the reference's camera pipeline spec -- TEST
 * INFRASTRUCTURE ONLY (the oracle; nothing in the product links it).
 *
 * Follows sandbox/apps/python/img_proc/campipe/polymage_campipe.py:13-304
 * with the C semantics the reference's generated code has: int arithmetic
 * with C promotion, truncating '/', stores converted to each stage's element
 * type (int16 for the demosaic stages, int for the matrix, uint8 for the
 * curve), Max/Min as selects (sandbox/constructs.py:312-319), and float
 * literals as double (sandbox/targetc.py:80-86).  Every function is computed
 * over its whole domain (all campipe functions are total).
 *
 * campipe_tables() builds the const functions (colour matrix and curve LUT)
 * exactly as the reference's expressions read; campipe() runs the pipeline.
 * OpenMP parallelizes the row loops when compiled with -fopenmp (the CPU
 * baseline build); results do not depend on the thread count.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef short s16;

#define SELMAX(a, b) ((a) > (b) ? (a) : (b))   /* Max(a, b) */
#define SELMIN(a, b) ((a) < (b) ? (a) : (b))   /* Min(a, b) */

/* matrix(x, y) = (int)((m3200(x,y)*alpha + m7000(x,y)*(1 - alpha)) * 256.0)
 * (:243-252); the constants 1.0/3200 and 1.0/7000 - 1.0/3200 are folded by
 * Python before code generation, so they appear here as those doubles. */
void campipe_matrix(float colour_temp, const float* m3200,
                    const float* m7000, int* mat) {
  for (int x = 0; x <= 2; ++x)
    for (int y = 0; y <= 3; ++y) {
      double alpha = ((1.0 / colour_temp) - 0.0003125) /
                     (0.00014285714285714287 - 0.0003125);
      mat[x * 4 + y] = (int)((((m3200[x * 4 + y] * alpha) +
                               (m7000[x * 4 + y] * (1 - alpha)))) * 256.0);
    }
}

/* curveLUT(v), v in [-32768, 32767] (:269-300) */
void campipe_curve(float gamma, float contrast, unsigned char* lut) {
  for (int v = -32768; v <= 32767; ++v) {
    float xf0 = (float)(v / 1024.0);
    double xf1 = (1.0 < xf0) ? 1.0 : xf0;            /* Min(1.0, xf) */
    double xf = (0.0 > xf1) ? 0.0 : xf1;              /* Max(0.0, xf) */
    float g = powf(xf, (1.0 / gamma));
    double b = 2.0 - powf(2.0, (contrast / 100.0));
    double a = 2.0 - (2.0 * b);
    double z = (g > 0.5)
                   ? (1.0 - (((a * (1.0 - g)) * (1.0 - g)) + (b * (1.0 - g))))
                   : (((a * g) * g) + (b * g));
    double t = z * 256.0;
    double t1 = (t > 0.0) ? t : 0.0;                  /* Max(z*256, 0) */
    double t2 = (t1 < 255.0) ? t1 : 255.0;            /* Min(., 255) */
    lut[v + 32768] = (unsigned char)t2;
  }
}

void campipe_tables(float colour_temp, float contrast, float gamma,
                    const float* m3200, const float* m7000, int* mat,
                    unsigned char* lut) {
  campipe_matrix(colour_temp, m3200, m7000, mat);
  campipe_curve(gamma, contrast, lut);
}

/* A function stored over [x0, x1] x [y0, y1] */
typedef struct {
  int x0, x1, y0, y1, w;
  s16* d;
} plane_t;

static plane_t mk(int x0, int x1, int y0, int y1) {
  plane_t p;
  p.x0 = x0; p.x1 = x1; p.y0 = y0; p.y1 = y1;
  p.w = y1 - y0 + 1;
  long n = (long)(x1 - x0 + 1) * p.w;
  p.d = (s16*)calloc(n > 0 ? n : 1, sizeof(s16));
  return p;
}
#define AT(p, x, y) ((p).d[(long)((x) - (p).x0) * (p).w + ((y) - (p).y0)])

/* img: int16 [R][C]; out: uint8 [3][R-48][C-64] */
void campipe(int R, int C, float colour_temp, float contrast, float gamma,
             const s16* img, const float* m3200, const float* m7000,
             unsigned char* out) {
  int mat[12];
  unsigned char* lut = (unsigned char*)malloc(65536);
  campipe_tables(colour_temp, contrast, gamma, m3200, m7000, mat, lut);
#define IMG(x, y) img[(long)(x) * C + (y)]
  /* intervals (:41-62) */
  const int h2x0 = 4, h2x1 = (R - 24 - 12) / 2 + 2;
  const int h2y0 = 6, h2y1 = (C - 32 - 16) / 2 + 2;
  const int h1x0 = 5, h1x1 = (R - 24 - 12) / 2 + 1;
  const int h1y0 = 7, h1y1 = (C - 32 - 16) / 2 + 1;
  const int h0x0 = 6, h0x1 = (R - 24 - 12) / 2;
  const int h0y0 = 8, h0y1 = (C - 32 - 16) / 2;
  const int g0x0 = 12, g0x1 = R - 24 - 12 - 1;
  const int g0y0 = 16, g0y1 = C - 32 - 16 - 1;

  /* 1. hot-pixel suppression on ghost_zone_2 (:72-83) */
  plane_t den = mk(8, R - 24 - 12 + 6 - 1, 12, C - 32 - 16 + 6 - 1);
#pragma omp parallel for
  for (int x = den.x0; x <= den.x1; ++x)
    for (int y = den.y0; y <= den.y1; ++y) {
      int x_max = SELMAX(IMG(x - 2, y), IMG(x + 2, y));
      int y_max = SELMAX(IMG(x, y - 2), IMG(x, y + 2));
      int x_min = SELMIN(IMG(x - 2, y), IMG(x + 2, y));
      int y_min = SELMIN(IMG(x, y - 2), IMG(x, y + 2));
      int mx = SELMAX(x_max, y_max), mn = SELMIN(x_min, y_min);
      int cl = SELMIN(mx, (int)IMG(x, y));
      cl = SELMAX(mn, cl);
      AT(den, x, y) = (s16)cl;
    }
  /* 2. deinterleave (:86-92) into the four planes */
  plane_t g_gr = mk(h2x0, h2x1, h2y0, h2y1), r_r = mk(h2x0, h2x1, h2y0, h2y1);
  plane_t b_b = mk(h2x0, h2x1, h2y0, h2y1), g_gb = mk(h2x0, h2x1, h2y0, h2y1);
#pragma omp parallel for
  for (int x = h2x0; x <= h2x1; ++x)
    for (int y = h2y0; y <= h2y1; ++y) {
      AT(g_gr, x, y) = AT(den, 2 * x, 2 * y);
      AT(r_r, x, y) = AT(den, 2 * x, 2 * y + 1);
      AT(b_b, x, y) = AT(den, 2 * x + 1, 2 * y);
      AT(g_gb, x, y) = AT(den, 2 * x + 1, 2 * y + 1);
    }
#define ABSD(a, b) ((a) > (b) ? (a) - (b) : (b) - (a))
  /* 3. green at red and blue sites (:118-140) */
  plane_t g_r = mk(h1x0, h1x1, h1y0, h1y1), g_b = mk(h1x0, h1x1, h1y0, h1y1);
#pragma omp parallel for
  for (int x = h1x0; x <= h1x1; ++x)
    for (int y = h1y0; y <= h1y1; ++y) {
      int gv_r = (AT(g_gb, x - 1, y) + AT(g_gb, x, y)) / 2;
      int gvd_r = ABSD(AT(g_gb, x - 1, y), AT(g_gb, x, y));
      int gh_r = (AT(g_gr, x, y + 1) + AT(g_gr, x, y)) / 2;
      int ghd_r = ABSD(AT(g_gr, x, y + 1), AT(g_gr, x, y));
      AT(g_r, x, y) = (s16)(ghd_r < gvd_r ? gh_r : gv_r);
      int gv_b = (AT(g_gr, x + 1, y) + AT(g_gr, x, y)) / 2;
      int gvd_b = ABSD(AT(g_gr, x + 1, y), AT(g_gr, x, y));
      int gh_b = (AT(g_gb, x, y - 1) + AT(g_gb, x, y)) / 2;
      int ghd_b = ABSD(AT(g_gb, x, y - 1), AT(g_gb, x, y));
      AT(g_b, x, y) = (s16)(ghd_b < gvd_b ? gh_b : gv_b);
    }
  /* red/blue at green sites, red at blue, blue at red (:148-212) */
  plane_t r_gr = mk(h0x0, h0x1, h0y0, h0y1), b_gr = mk(h0x0, h0x1, h0y0, h0y1);
  plane_t r_gb = mk(h0x0, h0x1, h0y0, h0y1), b_gb = mk(h0x0, h0x1, h0y0, h0y1);
  plane_t r_b = mk(h0x0, h0x1, h0y0, h0y1), b_r = mk(h0x0, h0x1, h0y0, h0y1);
#pragma omp parallel for
  for (int x = h0x0; x <= h0x1; ++x)
    for (int y = h0y0; y <= h0y1; ++y) {
      AT(r_gr, x, y) = (s16)(AT(g_gr, x, y) -
                             (AT(g_r, x, y) + AT(g_r, x, y - 1)) / 2 +
                             (AT(r_r, x, y - 1) + AT(r_r, x, y)) / 2);
      AT(b_gr, x, y) = (s16)(AT(g_gr, x, y) -
                             (AT(g_b, x, y) + AT(g_b, x - 1, y)) / 2 +
                             (AT(b_b, x, y) + AT(b_b, x - 1, y)) / 2);
      AT(r_gb, x, y) = (s16)(AT(g_gb, x, y) -
                             (AT(g_r, x, y) + AT(g_r, x + 1, y)) / 2 +
                             (AT(r_r, x, y) + AT(r_r, x + 1, y)) / 2);
      AT(b_gb, x, y) = (s16)(AT(g_gb, x, y) -
                             (AT(g_b, x, y) + AT(g_b, x, y + 1)) / 2 +
                             (AT(b_b, x, y) + AT(b_b, x, y + 1)) / 2);
      {
        int corr = AT(g_b, x, y) - (AT(g_r, x, y) + AT(g_r, x + 1, y - 1)) / 2;
        int rp = corr + (AT(r_r, x, y) + AT(r_r, x + 1, y - 1)) / 2;
        int rpd = ABSD(AT(r_r, x, y), AT(r_r, x + 1, y - 1));
        corr = AT(g_b, x, y) - (AT(g_r, x, y - 1) + AT(g_r, x + 1, y)) / 2;
        int rn = corr + (AT(r_r, x, y - 1) + AT(r_r, x + 1, y)) / 2;
        int rnd = ABSD(AT(r_r, x, y - 1), AT(r_r, x + 1, y));
        AT(r_b, x, y) = (s16)(rpd < rnd ? rp : rn);
      }
      {
        int corr = AT(g_r, x, y) - (AT(g_b, x, y) + AT(g_b, x - 1, y + 1)) / 2;
        int bp = corr + (AT(b_b, x, y) + AT(b_b, x - 1, y + 1)) / 2;
        int bpd = ABSD(AT(b_b, x, y), AT(b_b, x - 1, y + 1));
        corr = AT(g_r, x, y) - (AT(g_b, x, y + 1) + AT(g_b, x - 1, y)) / 2;
        int bn = corr + (AT(b_b, x, y + 1) + AT(b_b, x - 1, y)) / 2;
        int bnd = ABSD(AT(b_b, x, y + 1), AT(b_b, x - 1, y));
        AT(b_r, x, y) = (s16)(bpd < bnd ? bp : bn);
      }
    }
  /* 4. interleave (:215-235) and 5. colour correction (:254-262),
   * 6. curve (:294-300) */
  const int OH = g0x1 - g0x0 + 1, OW = g0y1 - g0y0 + 1;
#define IY(a, b, x, yy) (((yy) % 2 == 0) ? AT(a, x, (yy) / 2) : AT(b, x, (yy) / 2))
#define IXY(a1, b1, a2, b2, xx, yy) \
  (((xx) % 2 == 0) ? (s16)IY(a1, b1, (xx) / 2, yy) : (s16)IY(a2, b2, (xx) / 2, yy))
#pragma omp parallel for
  for (int x = g0x0; x <= g0x1; ++x)
    for (int y = g0y0; y <= g0y1; ++y) {
      s16 red = IXY(r_gr, r_r, r_b, r_gb, x, y);
      s16 green = IXY(g_gr, g_r, g_b, g_gb, x, y);
      s16 blue = IXY(b_gr, b_r, b_b, b_gb, x, y);
      int r = mat[3] + mat[0] * red + mat[1] * green + mat[2] * blue;
      int g = mat[7] + mat[4] * red + mat[5] * green + mat[6] * blue;
      int b = mat[11] + mat[8] * red + mat[9] * green + mat[10] * blue;
      s16 cr = (s16)(r / 256), cg = (s16)(g / 256), cb = (s16)(b / 256);
      long o = (long)(x - g0x0) * OW + (y - g0y0);
      out[0 * (long)OH * OW + o] = lut[cb + 32768];
      out[1 * (long)OH * OW + o] = lut[cg + 32768];
      out[2 * (long)OH * OW + o] = lut[cr + 32768];
    }
  free(den.d); free(g_gr.d); free(r_r.d); free(b_b.d); free(g_gb.d);
  free(g_r.d); free(g_b.d); free(r_gr.d); free(b_gr.d); free(r_gb.d);
  free(b_gb.d); free(r_b.d); free(b_r.d); free(lut);
}
