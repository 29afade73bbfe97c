// Checkpoint and trajectory files in the reference's formats (output.hpp).
// Host code only, apart from the device snapshot copies.
#include <cstring>
#include <utility>

#include "orrery_b200.h"
#include "output.hpp"
#include "system.hpp"

static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__,
              "reals are written as their in-memory bytes, which must be little-endian");

namespace ob {
namespace {

constexpr char kCheckpointMagic[8] = {'O', 'R', 'R', 'E', 'R', 'Y', 'C', 'K'};
constexpr char kTrajectoryMagic[8] = {'O', 'R', 'R', 'E', 'R', 'Y', 'T', 'J'};
constexpr uint32_t kFormatVersion = 1;
// Header flags (src/sim/checkpoint.cpp, src/sim/trajectory.cpp): bit 0 marks
// a single-precision build, bit 1 a trajectory that carries velocities.
constexpr uint32_t kFlagSinglePrecision = 1u << 0;
constexpr uint32_t kFlagHasVelocities = 1u << 1;
// Bounds a reader applies before sizing anything from a header, as the
// reference's readers do: 2^40 particles, 1 MiB of configuration text.
constexpr uint64_t kParticleLimit = 1ull << 40;
constexpr uint64_t kConfigurationLimit = 1ull << 20;

constexpr uint64_t kFnvBasis = 0xcbf29ce484222325ull;
constexpr uint64_t kFnvPrime = 0x00000100000001b3ull;

uint64_t fnv1a(uint64_t h, const unsigned char *p, size_t count) {
    for (size_t k = 0; k < count; ++k) {
        h = (h ^ p[k]) * kFnvPrime;
    }
    return h;
}

[[noreturn]] void fail(const std::string &path, const std::string &what) {
    throw Error(OB_ERROR_IO, path + ": " + what);
}

// Reads a file through the same checksum; a short read marks it failed and
// adds nothing to the checksum.
class ChecksumReader {
public:
    explicit ChecksumReader(std::FILE *file) : file_(file) {}
    bool bytes(void *data, size_t count) {
        if (!ok_ || std::fread(data, 1, count, file_) != count) {
            ok_ = false;
            return false;
        }
        sum_ = fnv1a(sum_, static_cast<const unsigned char *>(data), count);
        return true;
    }
    uint32_t u32() {
        unsigned char b[4] = {};
        bytes(b, 4);
        return static_cast<uint32_t>(b[0]) | static_cast<uint32_t>(b[1]) << 8 |
               static_cast<uint32_t>(b[2]) << 16 | static_cast<uint32_t>(b[3]) << 24;
    }
    uint64_t u64() {
        unsigned char b[8] = {};
        bytes(b, 8);
        uint64_t v = 0;
        for (int k = 7; k >= 0; --k) {
            v = v << 8 | b[k];
        }
        return v;
    }
    // The stored checksum, read without adding it to the running one.
    uint64_t stored_checksum() {
        const uint64_t expected = sum_;
        const uint64_t stored = u64();
        sum_ = expected;
        return stored;
    }
    [[nodiscard]] uint64_t checksum() const { return sum_; }
    [[nodiscard]] bool ok() const { return ok_; }

private:
    std::FILE *file_;
    uint64_t sum_ = kFnvBasis;
    bool ok_ = true;
};

struct FileCloser {
    std::FILE *file;
    ~FileCloser() {
        if (file != nullptr) {
            std::fclose(file);
        }
    }
};

} // namespace

// ---------------------------------------------------------------------------
// ChecksumWriter
// ---------------------------------------------------------------------------

void ChecksumWriter::bytes(const void *data, size_t count) {
    sum_ = fnv1a(sum_, static_cast<const unsigned char *>(data), count);
    if (ok_ && count > 0 && std::fwrite(data, 1, count, file_) != count) {
        ok_ = false;
    }
}

void ChecksumWriter::u32(uint32_t v) {
    const unsigned char b[4] = {static_cast<unsigned char>(v), static_cast<unsigned char>(v >> 8),
                                static_cast<unsigned char>(v >> 16),
                                static_cast<unsigned char>(v >> 24)};
    bytes(b, 4);
}

void ChecksumWriter::u64(uint64_t v) {
    unsigned char b[8];
    for (int k = 0; k < 8; ++k) {
        b[k] = static_cast<unsigned char>(v >> (8 * k));
    }
    bytes(b, 8);
}

void ChecksumWriter::string(const std::string &text) {
    u32(static_cast<uint32_t>(text.size()));
    bytes(text.data(), text.size());
}

void ChecksumWriter::close_section() {
    const uint64_t sum = sum_;
    u64(sum);
    sum_ = kFnvBasis;
}

// ---------------------------------------------------------------------------
// Checkpoints: magic, version, flags, step, particle count, configuration
// text, m x y z vx vy vz ax ay az, checksum (src/sim/checkpoint.cpp).
// ---------------------------------------------------------------------------

void write_checkpoint_file(const std::string &path, uint64_t step,
                           const std::string &configuration, uint64_t n,
                           const double *const arrays[kCheckpointArrays]) {
    if (configuration.size() > kConfigurationLimit) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "the configuration text exceeds 1 MiB");
    }
    for (int k = 0; k < kCheckpointArrays; ++k) {
        if (n > 0 && arrays[k] == nullptr) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "a checkpoint needs all ten state arrays");
        }
    }
    // Written beside the target and renamed over it, so a reader sees the old
    // checkpoint or the new one, never half of either.
    const std::string partial = path + ".partial";
    std::FILE *file = std::fopen(partial.c_str(), "wb");
    if (file == nullptr) {
        fail(partial, "could not be opened for writing");
    }
    bool ok;
    {
        ChecksumWriter w(file);
        w.bytes(kCheckpointMagic, sizeof kCheckpointMagic);
        w.u32(kFormatVersion);
        w.u32(0); // FP64 state: no single-precision flag
        w.u64(step);
        w.u64(n);
        w.string(configuration);
        for (int k = 0; k < kCheckpointArrays; ++k) {
            w.reals(arrays[k], n);
        }
        w.close_section();
        ok = w.ok() && std::fflush(file) == 0;
    }
    ok = (std::fclose(file) == 0) && ok;
    if (!ok) {
        std::remove(partial.c_str());
        fail(partial, "could not be written");
    }
    if (std::rename(partial.c_str(), path.c_str()) != 0) {
        std::remove(partial.c_str());
        fail(path, "could not be replaced by the new checkpoint");
    }
}

CheckpointHeader read_checkpoint_file(const std::string &path, double *const *arrays,
                                      uint64_t expected_n) {
    FileCloser closer{std::fopen(path.c_str(), "rb")};
    if (closer.file == nullptr) {
        fail(path, "could not be opened for reading");
    }
    ChecksumReader r(closer.file);
    char magic[8] = {};
    if (!r.bytes(magic, sizeof magic) || std::memcmp(magic, kCheckpointMagic, 8) != 0) {
        fail(path, "is not an ORRERYCK checkpoint");
    }
    const uint32_t version = r.u32();
    if (r.ok() && version != kFormatVersion) {
        fail(path, "is format version " + std::to_string(version) + "; version 1 is read here");
    }
    const uint32_t flags = r.u32();
    if (r.ok() && (flags & ~kFlagSinglePrecision) != 0) {
        fail(path, "sets header flags this reader does not know");
    }
    if (r.ok() && (flags & kFlagSinglePrecision) != 0) {
        fail(path, "holds single-precision state; these systems are FP64");
    }
    CheckpointHeader h;
    h.step = r.u64();
    h.n = r.u64();
    if (!r.ok() || h.n > kParticleLimit) {
        fail(path, "has an unreadable header");
    }
    const uint32_t length = r.u32();
    if (!r.ok() || length > kConfigurationLimit) {
        fail(path, "has an unreadable configuration");
    }
    h.configuration.resize(length);
    if (length > 0 && !r.bytes(&h.configuration[0], length)) {
        fail(path, "has an unreadable configuration");
    }
    if (arrays == nullptr) {
        return h;
    }
    if (h.n != expected_n) {
        throw Error(OB_ERROR_INVALID_ARGUMENT,
                    path + ": holds " + std::to_string(h.n) + " particles, not " +
                        std::to_string(expected_n));
    }
    for (int k = 0; k < kCheckpointArrays; ++k) {
        if (h.n > 0 && !r.bytes(arrays[k], h.n * sizeof(double))) {
            fail(path, "ends before its state is complete");
        }
    }
    const uint64_t stored = r.stored_checksum();
    if (!r.ok()) {
        fail(path, "ends before its state is complete");
    }
    if (stored != r.checksum()) {
        fail(path, "does not match its checksum (damaged, or written by an interrupted run)");
    }
    return h;
}

// ---------------------------------------------------------------------------
// Trajectories: header = magic, version, flags, particle count, timestep,
// masses, checksum; frame = step, time, x y z [vx vy vz], checksum
// (src/sim/trajectory.cpp).
// ---------------------------------------------------------------------------

TrajectoryFile::TrajectoryFile(const std::string &path, uint64_t n, const double *masses,
                               double timestep, bool with_velocities)
    : path_(path), n_(n), with_velocities_(with_velocities) {
    if (n > 0 && masses == nullptr) {
        throw Error(OB_ERROR_INVALID_ARGUMENT, "a trajectory header needs the masses");
    }
    file_ = std::fopen(path.c_str(), "wb");
    if (file_ == nullptr) {
        fail(path, "could not be opened for writing");
    }
    ChecksumWriter w(file_);
    w.bytes(kTrajectoryMagic, sizeof kTrajectoryMagic);
    w.u32(kFormatVersion);
    w.u32(with_velocities ? kFlagHasVelocities : 0u);
    w.u64(n);
    w.real(timestep);
    w.reals(masses, n);
    w.close_section();
    if (!w.ok()) {
        std::fclose(file_);
        file_ = nullptr;
        fail(path, "could not be written");
    }
}

TrajectoryFile::~TrajectoryFile() {
    if (file_ != nullptr) {
        std::fclose(file_);
    }
}

uint64_t TrajectoryFile::frame_checksum(uint64_t step, double time, const double *const xyz[3],
                                        const double *const v[3]) const {
    unsigned char head[16];
    for (int k = 0; k < 8; ++k) {
        head[k] = static_cast<unsigned char>(step >> (8 * k));
    }
    std::memcpy(head + 8, &time, 8);
    uint64_t h = fnv1a(kFnvBasis, head, sizeof head);
    for (int c = 0; c < 3; ++c) {
        h = fnv1a(h, reinterpret_cast<const unsigned char *>(xyz[c]), n_ * sizeof(double));
    }
    if (with_velocities_) {
        for (int c = 0; c < 3; ++c) {
            h = fnv1a(h, reinterpret_cast<const unsigned char *>(v[c]), n_ * sizeof(double));
        }
    }
    return h;
}

void TrajectoryFile::append_frame(uint64_t step, double time, const double *const xyz[3],
                                  const double *const v[3], uint64_t checksum) {
    unsigned char head[16];
    for (int k = 0; k < 8; ++k) {
        head[k] = static_cast<unsigned char>(step >> (8 * k));
    }
    std::memcpy(head + 8, &time, 8);
    unsigned char tail[8];
    for (int k = 0; k < 8; ++k) {
        tail[k] = static_cast<unsigned char>(checksum >> (8 * k));
    }
    const size_t bytes = n_ * sizeof(double);
    bool ok = std::fwrite(head, 1, sizeof head, file_) == sizeof head;
    for (int c = 0; c < 3 && ok && bytes > 0; ++c) {
        ok = std::fwrite(xyz[c], 1, bytes, file_) == bytes;
    }
    for (int c = 0; c < 3 && ok && bytes > 0 && with_velocities_; ++c) {
        ok = std::fwrite(v[c], 1, bytes, file_) == bytes;
    }
    ok = ok && std::fwrite(tail, 1, sizeof tail, file_) == sizeof tail;
    if (!ok) {
        fail(path_, "could not be written (frame " + std::to_string(frames_) + ")");
    }
    ++frames_;
}

void TrajectoryFile::flush() {
    if (std::fflush(file_) != 0) {
        fail(path_, "could not be flushed");
    }
}

// ---------------------------------------------------------------------------
// DeviceTrajectory
// ---------------------------------------------------------------------------

namespace {
// Writers checksum frames side by side; one more staging slot than writers
// lets the next snapshot land while every writer is busy.
constexpr int kTrajectoryWriters = 4;
constexpr int kTrajectorySlots = kTrajectoryWriters + 1;

std::vector<double> download_masses(System &system) {
    std::vector<double> m(system.size());
    system.synchronize();
    if (!m.empty()) {
        check(cudaMemcpy(m.data(), system.array(System::kM), sizeof(double) * m.size(),
                         cudaMemcpyDeviceToHost),
              "downloading masses");
    }
    return m;
}
} // namespace

DeviceTrajectory::DeviceTrajectory(const std::string &path, System &system, double timestep,
                                   bool with_velocities)
    : file_(path, system.size(), download_masses(system).data(), timestep, with_velocities),
      system_(&system), n_(system.size()), components_(with_velocities ? 6 : 3) {
    int device = 0;
    check(cudaGetDevice(&device), "cudaGetDevice");
    const size_t count = static_cast<size_t>(components_) * (n_ == 0 ? 1 : n_);
    slots_.resize(kTrajectorySlots);
    try {
        for (Slot &s : slots_) {
            s.device.reserve(count);
            check(cudaMallocHost(&s.host, count * sizeof(double)), "pinned staging");
            check(cudaEventCreateWithFlags(&s.landed, cudaEventDisableTiming), "an event");
        }
        for (int w = 0; w < kTrajectoryWriters; ++w) {
            cudaStream_t stream = nullptr;
            check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "a copy stream");
            copy_streams_.push_back(stream);
        }
        for (int w = 0; w < kTrajectoryWriters; ++w) {
            const cudaStream_t stream = copy_streams_[w];
            writers_.emplace_back([this, device, stream] {
                cudaSetDevice(device);
                run(stream);
            });
        }
    } catch (...) {
        stop_writers();
        throw;
    }
}

void DeviceTrajectory::stop_writers() noexcept {
    {
        std::lock_guard<std::mutex> lock(mutex_);
        stopping_ = true;
    }
    changed_.notify_all();
    for (std::thread &t : writers_) {
        t.join();
    }
    writers_.clear();
    for (Slot &s : slots_) {
        if (s.host != nullptr) {
            cudaFreeHost(s.host);
            s.host = nullptr;
        }
        if (s.landed != nullptr) {
            cudaEventDestroy(s.landed);
            s.landed = nullptr;
        }
    }
    for (cudaStream_t stream : copy_streams_) {
        cudaStreamDestroy(stream);
    }
    copy_streams_.clear();
}

DeviceTrajectory::~DeviceTrajectory() { stop_writers(); }

void DeviceTrajectory::raise_if_failed() {
    std::lock_guard<std::mutex> lock(mutex_);
    if (failure_code_ != 0) {
        throw Error(failure_code_, failure_);
    }
}

void DeviceTrajectory::write_frame(uint64_t step, double time) {
    raise_if_failed();
    int slot = -1;
    {
        std::unique_lock<std::mutex> lock(mutex_);
        changed_.wait(lock, [this] {
            for (const Slot &s : slots_) {
                if (!s.busy) {
                    return true;
                }
            }
            return false;
        });
        for (int k = 0; k < kTrajectorySlots; ++k) {
            if (!slots_[k].busy) {
                slot = k;
                break;
            }
        }
        slots_[slot].busy = true;
    }
    Slot &s = slots_[slot];
    try {
        // x y z (and vx vy vz) are contiguous in the system's state: one copy
        // each, in stream order between the steps around this call.
        const cudaStream_t stream = system_->stream();
        if (n_ > 0) {
            check(cudaMemcpyAsync(s.device.data(), system_->array(System::kX),
                                  3 * n_ * sizeof(double), cudaMemcpyDeviceToDevice, stream),
                  "snapshotting positions");
            if (components_ == 6) {
                check(cudaMemcpyAsync(s.device.data() + 3 * n_, system_->array(System::kVx),
                                      3 * n_ * sizeof(double), cudaMemcpyDeviceToDevice, stream),
                      "snapshotting velocities");
            }
        }
        check(cudaEventRecord(s.landed, stream), "recording a snapshot");
    } catch (...) {
        std::lock_guard<std::mutex> lock(mutex_);
        s.busy = false;
        changed_.notify_all();
        throw;
    }
    {
        std::lock_guard<std::mutex> lock(mutex_);
        queue_.push_back(Job{enqueued_++, slot, step, time, {}});
    }
    changed_.notify_all();
}

void DeviceTrajectory::write_host_frame(uint64_t step, double time, const double *const xyz[3],
                                        const double *const v[3]) {
    raise_if_failed();
    for (int c = 0; c < 3; ++c) {
        if (n_ > 0 && (xyz[c] == nullptr || (components_ == 6 && v[c] == nullptr))) {
            throw Error(OB_ERROR_INVALID_ARGUMENT, "a frame needs every array the file carries");
        }
    }
    std::vector<double> copy(static_cast<size_t>(components_) * n_);
    for (int c = 0; c < components_; ++c) {
        const double *src = c < 3 ? xyz[c] : v[c - 3];
        if (n_ > 0) {
            std::memcpy(copy.data() + c * n_, src, n_ * sizeof(double));
        }
    }
    {
        std::lock_guard<std::mutex> lock(mutex_);
        queue_.push_back(Job{enqueued_++, -1, step, time, std::move(copy)});
    }
    changed_.notify_all();
}

void DeviceTrajectory::run(cudaStream_t stream) {
    while (true) {
        Job job;
        {
            std::unique_lock<std::mutex> lock(mutex_);
            changed_.wait(lock, [this] { return stopping_ || !queue_.empty(); });
            if (queue_.empty()) {
                return; // stopping, nothing left
            }
            job = std::move(queue_.front());
            queue_.pop_front();
        }
        std::string error;
        int code = 0;
        const double *data = job.host.data();
        uint64_t checksum = 0;
        const double *xyz[3] = {nullptr, nullptr, nullptr};
        const double *v[3] = {nullptr, nullptr, nullptr};
        try {
            if (job.slot >= 0) {
                Slot &s = slots_[job.slot];
                check(cudaStreamWaitEvent(stream, s.landed, 0), "waiting for a snapshot");
                if (n_ > 0) {
                    check(cudaMemcpyAsync(s.host, s.device.data(),
                                          static_cast<size_t>(components_) * n_ * sizeof(double),
                                          cudaMemcpyDeviceToHost, stream),
                          "downloading a snapshot");
                }
                check(cudaStreamSynchronize(stream), "downloading a snapshot");
                data = s.host;
            }
            for (int c = 0; c < 3; ++c) {
                xyz[c] = data + c * n_;
                v[c] = data + (3 + c) * n_;
            }
            checksum = file_.frame_checksum(job.step, job.time, xyz, components_ == 6 ? v : nullptr);
        } catch (const Error &e) {
            code = e.code();
            error = e.what();
        } catch (const std::exception &e) {
            code = OB_ERROR_IO;
            error = e.what();
        }
        // Append in frame order; after a failure the file stops growing but
        // the order still advances, so no writer waits for a frame that will
        // never come.
        {
            std::unique_lock<std::mutex> lock(mutex_);
            changed_.wait(lock, [&] { return committed_ == job.sequence; });
            if (code == 0 && failure_code_ == 0) {
                try {
                    file_.append_frame(job.step, job.time, xyz, components_ == 6 ? v : nullptr,
                                       checksum);
                } catch (const Error &e) {
                    code = e.code();
                    error = e.what();
                } catch (const std::exception &e) {
                    code = OB_ERROR_IO;
                    error = e.what();
                }
            }
            if (code != 0 && failure_code_ == 0) {
                failure_code_ = code;
                failure_ = error;
            }
            if (job.slot >= 0) {
                slots_[job.slot].busy = false;
            }
            ++committed_;
        }
        changed_.notify_all();
    }
}

void DeviceTrajectory::flush() {
    {
        std::unique_lock<std::mutex> lock(mutex_);
        changed_.wait(lock, [this] { return committed_ == enqueued_; });
    }
    raise_if_failed();
    file_.flush();
}

uint64_t DeviceTrajectory::frames() {
    std::unique_lock<std::mutex> lock(mutex_);
    changed_.wait(lock, [this] { return committed_ == enqueued_; });
    return file_.frames();
}

} // namespace ob
