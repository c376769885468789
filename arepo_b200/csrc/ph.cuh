// ph.cuh -- 3-D Peano-Hilbert keys (126 bits: 42 levels x 3 bits).
//
// The curve is the reference's: peano_hilbert_key (src/domain/peano.c:374-390)
// driven by its 48-state tables rottable3/subpix3 (src/domain/peano.c:334-362).
// The table contents are data that must be identical for the keys (and hence the
// particle order and the node numbering) to be bit-exact; they are stored here
// packed as (next_state << 3 | digit), one 16-bit word per (state, octant).
#pragma once

#include <stdint.h>

namespace gg
{
// state transition, src/domain/peano.c:334-348 (rottable3)
static const unsigned char kPhRot[48][8] = {
    {36, 28, 25, 27, 10, 10, 25, 27}, {29, 11, 24, 24, 37, 11, 26, 26}, {8, 8, 25, 27, 30, 38, 25, 27},
    {9, 39, 24, 24, 9, 31, 26, 26},   {40, 24, 44, 32, 40, 6, 44, 6},   {25, 7, 33, 7, 41, 41, 45, 45},
    {4, 42, 4, 46, 26, 42, 34, 46},   {43, 43, 47, 47, 5, 27, 5, 35},   {33, 35, 36, 28, 33, 35, 2, 2},
    {32, 32, 29, 3, 34, 34, 37, 3},   {33, 35, 0, 0, 33, 35, 30, 38},   {32, 32, 1, 39, 34, 34, 1, 31},
    {24, 42, 32, 46, 14, 42, 14, 46}, {43, 43, 47, 47, 25, 15, 33, 15}, {40, 12, 44, 12, 40, 26, 44, 34},
    {13, 27, 13, 35, 41, 41, 45, 45}, {28, 41, 28, 22, 38, 43, 38, 22}, {42, 40, 23, 23, 29, 39, 29, 39},
    {41, 36, 20, 36, 43, 30, 20, 30}, {37, 31, 37, 31, 42, 40, 21, 21}, {28, 18, 28, 45, 38, 18, 38, 47},
    {19, 19, 46, 44, 29, 39, 29, 39}, {16, 36, 45, 36, 16, 30, 47, 30}, {37, 31, 37, 31, 17, 17, 46, 44},
    {12, 4, 1, 3, 34, 34, 1, 3},      {5, 35, 0, 0, 13, 35, 2, 2},      {32, 32, 1, 3, 6, 14, 1, 3},
    {33, 15, 0, 0, 33, 7, 2, 2},      {16, 0, 20, 8, 16, 30, 20, 30},   {1, 31, 9, 31, 17, 17, 21, 21},
    {28, 18, 28, 22, 2, 18, 10, 22},  {19, 19, 23, 23, 29, 3, 29, 11},  {9, 11, 12, 4, 9, 11, 26, 26},
    {8, 8, 5, 27, 10, 10, 13, 27},    {9, 11, 24, 24, 9, 11, 6, 14},    {8, 8, 25, 15, 10, 10, 25, 7},
    {0, 18, 8, 22, 38, 18, 38, 22},   {19, 19, 23, 23, 1, 39, 9, 39},   {16, 36, 20, 36, 16, 2, 20, 10},
    {37, 3, 37, 11, 17, 17, 21, 21},  {4, 17, 4, 46, 14, 19, 14, 46},   {18, 16, 47, 47, 5, 15, 5, 15},
    {17, 12, 44, 12, 19, 6, 44, 6},   {13, 7, 13, 7, 18, 16, 45, 45},   {4, 42, 4, 21, 14, 42, 14, 23},
    {43, 43, 22, 20, 5, 15, 5, 15},   {40, 12, 21, 12, 40, 6, 23, 6},   {13, 7, 13, 7, 41, 41, 22, 20}};

// key digit per octant, src/domain/peano.c:350-362 (subpix3)
static const unsigned char kPhSub[48][8] = {
    {0, 7, 1, 6, 3, 4, 2, 5}, {7, 4, 6, 5, 0, 3, 1, 2}, {4, 3, 5, 2, 7, 0, 6, 1}, {3, 0, 2, 1, 4, 7, 5, 6}, {1, 0, 6, 7, 2, 3, 5, 4},
    {0, 3, 7, 4, 1, 2, 6, 5}, {3, 2, 4, 5, 0, 1, 7, 6}, {2, 1, 5, 6, 3, 0, 4, 7}, {6, 1, 7, 0, 5, 2, 4, 3}, {1, 2, 0, 3, 6, 5, 7, 4},
    {2, 5, 3, 4, 1, 6, 0, 7}, {5, 6, 4, 7, 2, 1, 3, 0}, {7, 6, 0, 1, 4, 5, 3, 2}, {6, 5, 1, 2, 7, 4, 0, 3}, {5, 4, 2, 3, 6, 7, 1, 0},
    {4, 7, 3, 0, 5, 6, 2, 1}, {6, 7, 5, 4, 1, 0, 2, 3}, {7, 0, 4, 3, 6, 1, 5, 2}, {0, 1, 3, 2, 7, 6, 4, 5}, {1, 6, 2, 5, 0, 7, 3, 4},
    {2, 3, 1, 0, 5, 4, 6, 7}, {3, 4, 0, 7, 2, 5, 1, 6}, {4, 5, 7, 6, 3, 2, 0, 1}, {5, 2, 6, 1, 4, 3, 7, 0}, {7, 0, 6, 1, 4, 3, 5, 2},
    {0, 3, 1, 2, 7, 4, 6, 5}, {3, 4, 2, 5, 0, 7, 1, 6}, {4, 7, 5, 6, 3, 0, 2, 1}, {6, 7, 1, 0, 5, 4, 2, 3}, {7, 4, 0, 3, 6, 5, 1, 2},
    {4, 5, 3, 2, 7, 6, 0, 1}, {5, 6, 2, 1, 4, 7, 3, 0}, {1, 6, 0, 7, 2, 5, 3, 4}, {6, 5, 7, 4, 1, 2, 0, 3}, {5, 2, 4, 3, 6, 1, 7, 0},
    {2, 1, 3, 0, 5, 6, 4, 7}, {0, 1, 7, 6, 3, 2, 4, 5}, {1, 2, 6, 5, 0, 3, 7, 4}, {2, 3, 5, 4, 1, 0, 6, 7}, {3, 0, 4, 7, 2, 1, 5, 6},
    {1, 0, 2, 3, 6, 7, 5, 4}, {0, 7, 3, 4, 1, 6, 2, 5}, {7, 6, 4, 5, 0, 1, 3, 2}, {6, 1, 5, 2, 7, 0, 4, 3}, {5, 4, 6, 7, 2, 3, 1, 0},
    {4, 3, 7, 0, 5, 2, 6, 1}, {3, 2, 0, 1, 4, 5, 7, 6}, {2, 5, 1, 6, 3, 4, 0, 7}};

// Packed table for device code: entry [state*8 + octant] = next_state << 3 | digit.
struct PhTable
{
  uint16_t e[48 * 8];
};

static inline PhTable ph_make_table()
{
  PhTable t;
  for(int s = 0; s < 48; s++)
    for(int o = 0; o < 8; o++)
      t.e[s * 8 + o] = (uint16_t)((kPhRot[s][o] << 3) | kPhSub[s][o]);
  return t;
}

// 126-bit key from 42-bit integer coordinates; `tab` points to the packed table
// (shared or constant memory). Octant = (x bit) << 2 | (y bit) << 1 | (z bit), as
// in peano_hilbert_key.
__device__ __forceinline__ unsigned __int128 ph_key_dev(const uint16_t *tab, uint64_t x, uint64_t y, uint64_t z, int bits)
{
  unsigned state = 0;
  uint64_t hi = 0, lo = 0;
  for(int b = bits - 1; b >= 0; b--)
    {
      unsigned oct = (unsigned)((((x >> b) & 1) << 2) | (((y >> b) & 1) << 1) | ((z >> b) & 1));
      unsigned e   = tab[state * 8 + oct];
      hi           = (hi << 3) | (lo >> 61);
      lo           = (lo << 3) | (e & 7);
      state        = e >> 3;
    }
  return ((unsigned __int128)hi << 64) | lo;
}

// Low 3 bits of peano_hilbert_key(x, y, z, bits) (the digit of the finest level).
__device__ __forceinline__ int ph_last_digit_dev(const uint16_t *tab, uint64_t x, uint64_t y, uint64_t z, int bits)
{
  unsigned state = 0, digit = 0;
  for(int b = bits - 1; b >= 0; b--)
    {
      unsigned oct = (unsigned)((((x >> b) & 1) << 2) | (((y >> b) & 1) << 1) | ((z >> b) & 1));
      unsigned e   = tab[state * 8 + oct];
      digit        = e & 7;
      state        = e >> 3;
    }
  return (int)digit;
}
}  // namespace gg
