// Run output in the reference's file formats, from host arrays or from a
// device-resident system:
//   * ORRERYCK v1 checkpoints (write_checkpoint / read_checkpoint,
//     include/orrery/sim/checkpoint.hpp:85-94, src/sim/checkpoint.cpp);
//   * ORRERYTJ v1 trajectories (TrajectoryWriter,
//     include/orrery/sim/trajectory.hpp:112-146, src/sim/trajectory.cpp).
// Files are byte-identical to the reference's double-precision build's for the
// same state: every integer little-endian, every real its IEEE 754 bit
// pattern, each header and frame closed by the FNV-1a checksum of its bytes.
// The configuration a checkpoint carries is the caller's text (the reference
// writes it with sim::write_configuration); it is stored and returned as is.
#pragma once

#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#include "runtime.hpp"

namespace ob {

class System;

// A file written through a 64-bit FNV-1a checksum of every byte, the
// reference's checksum (include/orrery/sim/binary_stream.hpp:74-81).
class ChecksumWriter {
public:
    explicit ChecksumWriter(std::FILE *file) : file_(file) {}
    void bytes(const void *data, size_t count);
    void u32(uint32_t v);
    void u64(uint64_t v);
    void real(double v) { bytes(&v, sizeof v); } // little-endian host: the bit pattern
    void reals(const double *v, uint64_t count) { bytes(v, count * sizeof(double)); }
    void string(const std::string &text); // 32-bit length, then the bytes
    // Writes the checksum of everything so far (not itself checksummed) and
    // starts a new one, as a fresh reference BinaryWriter would.
    void close_section();
    [[nodiscard]] bool ok() const { return ok_; }

private:
    std::FILE *file_;
    uint64_t sum_ = 0xcbf29ce484222325ull;
    bool ok_ = true;
};

// The ten state arrays of a checkpoint, in the file's order:
// m, x, y, z, vx, vy, vz, ax, ay, az.
constexpr int kCheckpointArrays = 10;

void write_checkpoint_file(const std::string &path, uint64_t step,
                           const std::string &configuration, uint64_t n,
                           const double *const arrays[kCheckpointArrays]);

struct CheckpointHeader {
    uint64_t step = 0;
    uint64_t n = 0;
    std::string configuration;
};

// Reads and validates (magic, version, flags, sizes, checksum) a checkpoint.
// With `arrays` NULL only the header is read (the checksum is not checked).
CheckpointHeader read_checkpoint_file(const std::string &path,
                                      double *const *arrays /* kCheckpointArrays, or NULL */,
                                      uint64_t expected_n);

// An ORRERYTJ v1 file being written: the header at construction, then frames.
class TrajectoryFile {
public:
    TrajectoryFile(const std::string &path, uint64_t n, const double *masses, double timestep,
                   bool with_velocities);
    ~TrajectoryFile();
    TrajectoryFile(const TrajectoryFile &) = delete;
    TrajectoryFile &operator=(const TrajectoryFile &) = delete;

    // xyz: x, y, z (n each); v: vx, vy, vz, or NULL when the file carries no
    // velocities.
    void write_frame(uint64_t step, double time, const double *const xyz[3],
                     const double *const v[3]) {
        append_frame(step, time, xyz, v, frame_checksum(step, time, xyz, v));
    }
    // A frame's checksum (each frame has its own), and the frame's bytes with
    // that checksum: separate so that frames can be checksummed in parallel
    // and appended in order.
    [[nodiscard]] uint64_t frame_checksum(uint64_t step, double time, const double *const xyz[3],
                                          const double *const v[3]) const;
    void append_frame(uint64_t step, double time, const double *const xyz[3],
                      const double *const v[3], uint64_t checksum);
    void flush();
    [[nodiscard]] uint64_t frames() const noexcept { return frames_; }
    [[nodiscard]] uint64_t size() const noexcept { return n_; }
    [[nodiscard]] bool with_velocities() const noexcept { return with_velocities_; }

private:
    std::string path_;
    std::FILE *file_ = nullptr;
    uint64_t n_;
    bool with_velocities_;
    uint64_t frames_ = 0;
};

// Trajectory frames of a device-resident system, written without stalling
// its stream: a frame is a device-to-device snapshot of the positions (and
// velocities) into one of a few staging slots, enqueued on the system's
// stream. A pool of writer threads takes frames in order; each copies its
// slot to pinned host memory on its own stream once the snapshot has landed
// and checksums it (the checksum is a sequential byte chain, ~0.7 GB/s on one
// core, so frames are checksummed side by side), then appends it to the file
// in frame order. When every slot is in flight the next frame waits for one.
class DeviceTrajectory {
public:
    DeviceTrajectory(const std::string &path, System &system, double timestep,
                     bool with_velocities);
    ~DeviceTrajectory();
    DeviceTrajectory(const DeviceTrajectory &) = delete;
    DeviceTrajectory &operator=(const DeviceTrajectory &) = delete;

    void write_frame(uint64_t step, double time);
    // Host-array frames go through the same ordered queue.
    void write_host_frame(uint64_t step, double time, const double *const xyz[3],
                          const double *const v[3]);
    // Waits until every queued frame is in the file, then flushes it.
    void flush();
    [[nodiscard]] uint64_t frames();

private:
    struct Slot {
        DeviceArray<double> device;
        double *host = nullptr; // pinned
        cudaEvent_t landed = nullptr;
        bool busy = false;
    };
    struct Job {
        uint64_t sequence; // position in the file
        int slot;          // -1: the host copy in `host`
        uint64_t step;
        double time;
        std::vector<double> host;
    };
    void run(cudaStream_t stream);
    void raise_if_failed(); // rethrows a writer failure (caller holds no lock)
    void stop_writers() noexcept;

    TrajectoryFile file_;
    System *system_;
    uint64_t n_;
    int components_; // 3 or 6 arrays per frame
    std::vector<Slot> slots_;
    std::vector<cudaStream_t> copy_streams_; // one per writer
    std::mutex mutex_;
    std::condition_variable changed_;
    std::deque<Job> queue_;
    uint64_t enqueued_ = 0;   // frames given so far
    uint64_t committed_ = 0;  // frames appended (or skipped after a failure)
    bool stopping_ = false;
    std::string failure_;
    int failure_code_ = 0;
    std::vector<std::thread> writers_;
};

} // namespace ob
