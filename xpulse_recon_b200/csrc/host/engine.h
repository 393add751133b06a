// engine.h -- the reconstruction schedulers ("memory modes") on the C ABI.
//
// naive      reconstruction_n.hpp:27-88    everything resident on the device
// method_1a  reconstruction_lpln.hpp:27-96 volume streamed in y-slabs, one buffer, synchronous
// method_1b  reconstruction_lpla.hpp:29-157 volume streamed in y-slabs, double-buffered on
//                                          copy streams overlapped with the projector
// method_1c  reconstruction_lplh.hpp:40-219 as 1b with method_1c's semantics (first-iteration
//                                          volume 1/W, unweighted first error, NaN-skipping
//                                          back projection, every angle of the sub-iteration)
// method_2   reconstruction_chunk.hpp:36-131 independent slab chunks with padding against a
//                                          cropped detector-row window (geometry_chunk.hpp)
// simulate   reconstruction.hpp:66-158      forward_exec: 32 jittered samples of the saved
//                                          volume, cylinder mask, projections written as TIFF
#pragma once

#include <cstdint>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "../../../include/xpr.h"
#include "params.h"

namespace xpr {

// Source of the measured projections, in acquisition order.
struct ImageSource {
    virtual ~ImageSource() = default;
    virtual int64_t count() const = 0;
    virtual uint32_t width() const = 0;
    virtual uint32_t height() const = 0;
    virtual void read(int64_t i, float *dst) = 0;  // width*height floats
};

// The reference's input: every float32 TIFF of a directory, all of the first file's
// size (dataset.hpp:214-269); files are taken in lexicographic order (the reference
// uses directory order, which is unspecified).
std::unique_ptr<ImageSource> directory_images(const std::string &dir);
// Images already in host memory (count x height x width floats, acquisition order).
std::unique_ptr<ImageSource> memory_images(const float *data, int64_t count, uint32_t width, uint32_t height);

struct RunStats {
    double seconds_total = 0.0, seconds_iterations = 0.0;
    int64_t subiterations = 0;
    uint64_t pairs = 0;  // voxel x projection pairs processed by the projector
};

class Engine {
public:
    Engine(const Params &p, std::unique_ptr<ImageSource> images, bool write_files);
    ~Engine();
    Engine(const Engine &) = delete;
    Engine &operator=(const Engine &) = delete;

    // Results into `dst` (vwidth * vheight * vwidth floats, the caller's) instead of volume().
    void set_output(float *dst) { out_ = dst; }
    void reconstruct();       // exec() of the selected method
    void simulate();          // forward_exec() of the volume in the output directory
    const std::vector<float> &volume() const { return volume_; }
    const RunStats &stats() const { return stats_; }
    int64_t vwidth() const { return go_.vwidth; }
    int64_t vheight() const { return go_.vheight; }

private:
    struct Impl;
    std::unique_ptr<Impl> d_;
    Params p_;
    xpr_geom_params gp_{};
    xpr_geom_out go_{};
    std::vector<float> volume_;
    float *out_ = nullptr;
    RunStats stats_;
};

}  // namespace xpr
