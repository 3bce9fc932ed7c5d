// Host-side design helpers: receive window LUT, FIR filters, scan-conversion tables.
#pragma once

#include <stdint.h>

#include <vector>

#include "supra_b200.h"

namespace sb {

// Receive window sampled into n entries and normalised to its maximum (the LUT SUPRA's
// WindowFunction builds, Beamformer/WindowFunction.cpp:18-49 with the formulas of WindowFunction.h:121-138).
std::vector<float> windowLut(int type, float param, size_t n);

// Window-method FIR design (SupraLib/utilities/FirFilterFactory.h:58-230): type 0 low-pass,
// 1 high-pass, 2 band-pass, 3 Hilbert; window 0 rect, 1 Hann, 2 Hamming, 3 Kaiser (beta 4).
std::vector<float> firDesign(size_t length, int type, int window, double fs, double frequency, double bandwidth);

// Scan-conversion tables (Beamformer/ScanConverter.cu:513-894).
struct ScanTables {
    uint32_t size[3] = {0, 0, 0};
    double bbMin[3] = {0, 0, 0};
    std::vector<uint8_t> mask;
    std::vector<uint32_t> sampleIdx;
    std::vector<float> weightX, weightY, weightZ;
};
// Computes the image size; when `fill2D` the 2D tables too (host, double precision, serial order).
void scanGeometry(const sb_scanline_rx* lines, uint32_t lx, uint32_t ly, double depth, double resolution,
                  ScanTables& t);
void scanTables2D(const sb_scanline_rx* lines, uint32_t lx, uint32_t ly, uint32_t numSamples, double depth,
                  double resolution, ScanTables& t);

}  // namespace sb
