// Host-only check of the interior tiles' TMA halo boxes (compiled by nvcc,
// run on the CPU): for every grid and CPML width swept, every tile of the
// rectangle mhd_interior_rect returns must
//   - pass the kernels' own interior test (mhd_interior's condition),
//   - start its FP64 halo box at x0 - 6 >= 0 with (x0 - 6) * 8 a multiple of
//     16 bytes (a misaligned TMA x coordinate faults the GPU), y0 - 5 >= 0,
//   - keep its stencil footprint [x0-5, x0+37) x [y0-5, y0+13) inside the
//     grid and away from the CPML slabs, and
//   - read at most one column past the grid edge in the 44-wide box (TMA
//     fills it with zeros; the kernel never reads it).
// Prints "ok <tiles checked>" or the first violation; exit status 0 / 1.
#include <cstdio>

#include "../../sparc2_b200/csrc/mhd_body.cuh"

using namespace sparc;

int main() {
  long long tiles = 0;
  for (int nx = 32; nx <= 320; nx += 2)
    for (int ny = 16; ny <= 200; ny += 3)
      for (int np = 0; np <= 20; np += 4) {
        const int npa[4] = {np, np, np, np};
        int ix0, ix1, iy0, iy1;
        mhd_interior_rect(nx, ny, npa, ix0, ix1, iy0, iy1);
        const int xm = np > 5 ? np : 5, ym = xm;
        for (int tx = ix0; tx < ix1; ++tx)
          for (int ty = iy0; ty < iy1; ++ty) {
            const int x0 = tx * mg::TX, y0 = ty * mg::TY;
            const int hx = x0 - 5 - MhdBuf<double, true>::XOFF;
            bool ok = x0 >= xm && x0 + mg::TX <= nx - xm && y0 >= ym && y0 + mg::TY <= ny - ym;
            ok = ok && hx >= 0 && (hx * 8) % 16 == 0 && y0 - 5 >= 0;
            ok = ok && x0 - 5 >= 0 && x0 + mg::TX + 5 <= nx && y0 + mg::TY + 5 <= ny;
            ok = ok && hx + MhdBuf<double, true>::HXL <= nx + 1;
            if (!ok) {
              std::printf("violation nx=%d ny=%d np=%d tile x0=%d y0=%d\n", nx, ny, np, x0, y0);
              return 1;
            }
            ++tiles;
          }
      }
  std::printf("ok %lld\n", tiles);
  return 0;
}
