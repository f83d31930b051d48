// render.cpp -- headless images of simulated states (no graphics API): the
// reference viewer's two pictures of a state, as RGB bytes, and a binary PPM
// writer for them.
//
// grn_render_cells restates CellImageThread::calcImage
// (Src/UI/GUICommon/Simulator/cellimagethread.cpp:59-84): morphogens 0, 1, 2
// as red, green, blue, each 255 * min(1, c) truncated.
// grn_render_concentrations restates ConcentImageThread::calcImage
// (Src/UI/GUICommon/Simulator/concentimagethread.cpp:55-82): every product in
// use adds its palette colour (ColorsConfig::colorsMorp,
// Src/UI/GUICommon/Private/colorsconfig.cpp:11-31) times c / factor to an
// integer accumulator (truncated after each addition), clamped above at 255
// and packed as qRgb packs it (low 8 bits).

#include <cmath>
#include <cstdio>

#include "../../include/grn_gpu.h"

namespace {

// The viewer's product palette, 0xRRGGBB (same colours, same order).
const uint32_t kPalette[19] = {
    0xFF0000, 0x00FF00, 0x0000FF, 0xFF00FF, 0xFFFF00, 0x00FFFF, 0xC0C0C0,
    0x7425B1, 0xFF9233, 0xAD2323, 0xFED4D9, 0x5F6142, 0x43B3AE, 0xFEDA83,
    0x814A19, 0xC0D8F2, 0xC3C982, 0xE88F2B, 0x868A35};

// int(255 * min(1, c)) with the reference's min (MathAlgo::min keeps the
// first argument unless the second is smaller); NaN renders as 0.
int channel(double c) {
  const double v = 255.0 * (c < 1.0 ? c : 1.0);
  if (!(v == v)) return 0;
  return (int)(v < -2147483648.0 ? -2147483648.0 : v) & 0xff;
}

// int(acc + add), the reference's `int += double`, kept inside int range.
int add_trunc(int acc, double add) {
  const double v = acc + add;
  if (!(v == v)) return acc;
  return (int)(v > 2147483647.0 ? 2147483647.0 : v < -2147483648.0 ? -2147483648.0 : v);
}

}  // namespace

extern "C" {

grn_status grn_render_cells(const float *planes, int n_planes, int n_morphogens, int width,
                            int height, uint8_t *rgb) {
  if (!planes || !rgb || width < 1 || height < 1 || n_morphogens < 1 || n_morphogens > 3 ||
      n_planes < n_morphogens)
    return GRN_ERR_INVALID_ARGUMENT;
  const size_t cells = (size_t)width * height;
  for (size_t i = 0; i < cells; ++i) {
    uint8_t *px = rgb + 3 * i;
    px[0] = (uint8_t)channel(planes[i]);
    px[1] = n_morphogens > 1 ? (uint8_t)channel(planes[cells + i]) : 0;
    px[2] = n_morphogens > 2 ? (uint8_t)channel(planes[2 * cells + i]) : 0;
  }
  return GRN_OK;
}

grn_status grn_render_concentrations(const float *planes, int n_planes, int width, int height,
                                     double factor, uint8_t *rgb) {
  if (!planes || !rgb || width < 1 || height < 1 || n_planes < 0 || !(factor != 0.0))
    return GRN_ERR_INVALID_ARGUMENT;
  const size_t cells = (size_t)width * height;
  for (size_t i = 0; i < cells; ++i) {
    int r = 0, g = 0, b = 0;
    for (int k = 0; k < n_planes; ++k) {
      const double f = planes[k * cells + i] / factor;
      const uint32_t c = kPalette[k % 19];
      r = add_trunc(r, ((c >> 16) & 0xff) * f);
      g = add_trunc(g, ((c >> 8) & 0xff) * f);
      b = add_trunc(b, (c & 0xff) * f);
    }
    uint8_t *px = rgb + 3 * i;
    px[0] = (uint8_t)((r > 255 ? 255 : r) & 0xff);
    px[1] = (uint8_t)((g > 255 ? 255 : g) & 0xff);
    px[2] = (uint8_t)((b > 255 ? 255 : b) & 0xff);
  }
  return GRN_OK;
}

grn_status grn_write_ppm(const char *path, const uint8_t *rgb, int width, int height) {
  if (!path || !rgb || width < 1 || height < 1) return GRN_ERR_INVALID_ARGUMENT;
  FILE *f = std::fopen(path, "wb");
  if (!f) return GRN_ERR_INVALID_ARGUMENT;
  const size_t n = (size_t)width * height * 3;
  const bool ok = std::fprintf(f, "P6\n%d %d\n255\n", width, height) > 0 &&
                  std::fwrite(rgb, 1, n, f) == n;
  return (std::fclose(f) == 0 && ok) ? GRN_OK : GRN_ERR_INVALID_ARGUMENT;
}

}  // extern "C"
