// pygranite_module.cpp — the pygranite Python surface, rebuilt above the C ABI.
//
// Same module contents as the reference's binding (source/pygranite.cpp:41-152): the nine
// enums with their values and export_values() registration order, IntegratorSettings with
// its 21 fields and defaults (source/granite/IntegratorSettings.hpp:83-181), the DataLoader
// trampoline (source/granite/DataLoader.hpp:26-144), TrajectorySet and its accessors
// (source/granite/TrajectorySet.cpp) and TrajectoryIntegrator(settings, loader, set).compute().
// The host driver of the reference (TrajectoryIntegrator.cpp:146-360, .tpp:467-1049) is
// replaced by calls into libgranite_b200.so (include/granite_b200.h).
#include <pybind11/numpy.h>
#include <pybind11/pybind11.h>
#include <pybind11/stl.h>

#include <cstring>
#include <exception>
#include <memory>
#include <sstream>
#include <string>
#include <unordered_map>
#include <vector>

#include "copy_pool.h"

#include "../../include/granite_b200.h"

namespace py = pybind11;

namespace granite __attribute__((visibility("hidden"))) {

enum class Space : uint32_t { Space3D = 0, Space2D = 1 };
enum class Integrator : uint32_t { ExplicitEuler = 0, ClassicRungeKutta = 1 };
enum class BorderMode : uint32_t { Block = 0, LoopX = 1, LoopY = 2, LoopXY = 3 };
enum class CurvatureMode : uint32_t { Off = 0, TotalCurvature = 1, FastTotalCurvature = 2, IndividualAndTotalCurvature = 3 };
enum class AbortMode : uint32_t { Time = 0, Length = 1, FitLength = 2 };
enum class UpLiftMode : uint32_t { Off = 0, Constant = 1, Dynamic = 2 };
enum class WindfieldMode : uint32_t { Constant = 0, Dynamic = 1 };
enum class ConstantsMode : uint32_t { Off = 0, Constant = 1, Dynamic = 2 };
enum class AdditionalVolumeMode : uint32_t { Off = 0, Constant = 1, Dynamic = 2 };
enum class AbortReason : int32_t { Time = 0, Length = 1, Domain = 2, Topography = 3, Wind = 4 };
enum class WindStorage : int32_t { Float32 = 0, BFloat16 = 1, Float16 = 2 };

using farray = py::array_t<float, py::array::c_style | py::array::forcecast>;
using map_t = std::unordered_map<std::string, py::array_t<float>>;

[[noreturn]] void user_error(const std::string &msg) { throw std::runtime_error("ERROR < USER INPUT | " + msg + " >"); }

void user_warning(const std::string &msg) { py::print("WARNING < USER INPUT | " + msg + " >"); }

struct IntegratorSettings {
    float SphereRadius{0.f};
    granite::Space Space{granite::Space::Space3D};
    granite::Integrator Integrator{granite::Integrator::ClassicRungeKutta};
    granite::WindfieldMode WindfieldMode{granite::WindfieldMode::Dynamic};
    granite::ConstantsMode ConstantsMode{granite::ConstantsMode::Off};
    granite::AdditionalVolumeMode AdditionalVolumeMode{granite::AdditionalVolumeMode::Off};
    granite::UpLiftMode UpLiftMode{granite::UpLiftMode::Off};
    float DeltaT{1};
    float DataTimeDistance{60};
    std::vector<float> GridScale{25, 25, 25};
    std::vector<float> Offset{0, 0, 0};
    size_t SaveInterval{1};
    bool Reverse{false};
    granite::BorderMode BorderMode{granite::BorderMode::Block};
    granite::CurvatureMode CurvatureMode{granite::CurvatureMode::Off};
    float MaximumLength{0.f};
    float MaximumSimulationTime{100.f};
    granite::AbortMode AbortMode{granite::AbortMode::Time};
    int32_t MinimumAliveParticles{0};
    py::array_t<float> Topography = py::array_t<float>(0);
    std::vector<std::string> AdditionalCompute;
    // engine options beyond the reference
    granite::WindStorage WindStorage{granite::WindStorage::Float32};
    bool Float64Time{false};
    bool CompensatedPositions{false};
    int32_t RingSlots{0};
    int32_t StepsPerLaunch{0};
    int32_t SortInterval{-1};
    int32_t BlockSize{0};
    int32_t Device{0};
    int32_t WindLayout{0};
    bool PinnedResults{false};
    bool ReferenceFilter{false};
};

// float32 array of `shape` in page-locked host memory (gr_host_alloc); the block returns to the
// library's cache when the array is released.  The engine's uploads from, and result copies
// into, such arrays are single DMAs without staging copies.
py::array_t<float> pinned_empty(const std::vector<py::ssize_t> &shape) {
    size_t count = 1;
    for (auto d : shape) {
        if (d < 0) user_error("negative dimension");
        count *= static_cast<size_t>(d);
    }
    if (count == 0) return py::array_t<float>(shape);
    void *p = nullptr;
    if (gr_host_alloc(static_cast<int64_t>(count * sizeof(float)), &p) != GR_OK) throw std::runtime_error(gr_last_error());
    py::capsule owner(p, [](void *q) { gr_host_free(q); });
    return py::array_t<float>(shape, static_cast<float *>(p), owner);
}

class DataLoader {
  public:
    DataLoader() = default;
    virtual ~DataLoader() = default;
    virtual bool step() = 0;
    virtual std::vector<py::array_t<float>> windfield() = 0;
    virtual py::array_t<float> uplift() { return py::array_t<float>(); }
    virtual map_t constants() { return map_t(); }
    virtual map_t additionalVolumes() { return map_t(); }
};

class PyDataLoader : public DataLoader {
  public:
    using DataLoader::DataLoader;
    bool step() override { PYBIND11_OVERRIDE_PURE(bool, DataLoader, step); }
    std::vector<py::array_t<float>> windfield() override {
        PYBIND11_OVERRIDE_PURE(std::vector<py::array_t<float>>, DataLoader, windfield);
    }
    py::array_t<float> uplift() override { PYBIND11_OVERRIDE(py::array_t<float>, DataLoader, uplift); }
    map_t constants() override { PYBIND11_OVERRIDE(map_t, DataLoader, constants); }
    map_t additionalVolumes() override { PYBIND11_OVERRIDE(map_t, DataLoader, additionalVolumes); }
};

// Ordered string -> array view of a loader dictionary (Python dict order; the reference's
// std::unordered_map order is unspecified).
std::vector<std::pair<std::string, farray>> ordered(const map_t &m, py::object original) {
    std::vector<std::pair<std::string, farray>> out;
    if (py::isinstance<py::dict>(original)) {
        for (auto item : original.cast<py::dict>()) {
            std::string k = py::str(item.first);
            auto it = m.find(k);
            if (it != m.end()) out.emplace_back(k, farray::ensure(it->second));
        }
    } else {
        for (const auto &kv : m) out.emplace_back(kv.first, farray::ensure(kv.second));
    }
    return out;
}

class TrajectorySet {
  public:
    granite::Space space{granite::Space::Space2D};
    size_t n{0};
    size_t dim{2};
    py::array_t<float> traj;              // (n, L, dim)
    std::vector<AbortReason> abort_reasons;
    std::vector<float> total_curvature, lengths;
    py::array_t<float> curv;              // (n, Lc)
    std::vector<std::pair<std::string, py::array_t<float>>> volume_data;
    std::vector<py::array_t<float>> compute_data;
    size_t num_compute{0};
    int64_t particle_steps{0};            // of the run that produced this set (0 for seeds)

    TrajectorySet() = default;

    explicit TrajectorySet(py::array_t<float> points_in) {
        farray points = farray::ensure(points_in);
        if (!points || points.ndim() != 2) user_error("Currently only 1 dimensional initial pointsets are supported.");
        n = static_cast<size_t>(points.shape(0));
        if (points.shape(1) == 2) space = granite::Space::Space2D;
        else if (points.shape(1) == 3) space = granite::Space::Space3D;
        else user_error("TrajectorySet does not support the given type of coordinates.");
        dim = static_cast<size_t>(points.shape(1));
        traj = py::array_t<float>({static_cast<py::ssize_t>(n), py::ssize_t(1), static_cast<py::ssize_t>(dim)});
        if (n * dim) std::memcpy(traj.mutable_data(), points.data(), n * dim * sizeof(float));
        curv = py::array_t<float>({static_cast<py::ssize_t>(n), py::ssize_t(0)});
    }

    size_t records() const { return static_cast<size_t>(traj.shape(1)); }

    // last record, (n, dim) contiguous (the seeds of a following run, cpp:424-442)
    std::vector<float> last_points() const {
        std::vector<float> out(n * dim);
        const size_t L = records();
        const float *src = traj.data();
        for (size_t i = 0; i < n; ++i)
            for (size_t d = 0; d < dim; ++d) out[i * dim + d] = src[(i * L + (L - 1)) * dim + d];
        return out;
    }

    py::array_t<float> trajectory(size_t particle_id) const {
        const size_t L = records();
        py::array_t<float> out({static_cast<py::ssize_t>(L), static_cast<py::ssize_t>(dim)});
        if (particle_id >= n) throw py::index_error("particle id out of range");
        std::memcpy(out.mutable_data(), traj.data() + particle_id * L * dim, L * dim * sizeof(float));
        return out;
    }

    py::array_t<float> trajectories() const {
        py::array_t<float> out({static_cast<py::ssize_t>(n), static_cast<py::ssize_t>(records()), static_cast<py::ssize_t>(dim)});
        if (out.size()) granite_b200::parallel_memcpy(out.mutable_data(), traj.data(), out.size() * sizeof(float));
        return out;
    }

    py::array_t<float> cloud() const {
        py::array_t<float> out({static_cast<py::ssize_t>(n * records()), static_cast<py::ssize_t>(dim)});
        if (out.size()) granite_b200::parallel_memcpy(out.mutable_data(), traj.data(), out.size() * sizeof(float));
        return out;
    }

    static py::array_t<float> vec(const std::vector<float> &v) {
        py::array_t<float> out(static_cast<py::ssize_t>(v.size()));
        if (!v.empty()) std::memcpy(out.mutable_data(), v.data(), v.size() * sizeof(float));
        return out;
    }

    static py::array_t<float> copy2(const py::array_t<float> &a) {
        py::array_t<float> out({a.shape(0), a.shape(1)});
        if (out.size()) granite_b200::parallel_memcpy(out.mutable_data(), a.data(), out.size() * sizeof(float));
        return out;
    }

    py::array_t<float> totalCurvatures() const { return vec(total_curvature); }
    py::array_t<float> individualLengths() const { return vec(lengths); }
    py::array_t<float> curvatures() const { return copy2(curv); }

    py::array_t<float> volumeInfo(std::string key) const {
        for (const auto &kv : volume_data)
            if (kv.first == key) return copy2(kv.second);
        user_error("TrajectorySet: Volume with given key '" + key + "' does not exist!");
    }

    py::array_t<float> computeInfo(size_t id) const {
        if (id < num_compute && id < compute_data.size()) return copy2(compute_data[id]);
        user_error("TrajectorySet: Volume with given id does not exist!");
    }

    size_t lengthTrajectories() const { return records(); }
    size_t numberTrajectories() const { return n; }
    std::vector<AbortReason> abortReasons() const { return abort_reasons; }
};

class TrajectoryIntegrator {
  public:
    TrajectoryIntegrator(IntegratorSettings &settings, DataLoader &loader, TrajectorySet &set)
        : settings_(settings), loader_(loader) {
        // initSet (cpp:424-442): the last record of the given set seeds the run
        if (set.n == 0 && set.records() == 0) user_error("Provided TrajectorySet does not contain any data.");
        space_ = set.space;
        n_ = set.n;
        if (settings_.Space != space_) user_error("Dimensions of IntegratorSettings and provided TrajectorySet do not match.");
        dim_ = space_ == granite::Space::Space3D ? 3 : 2;
        seeds_ = set.last_points();
        create_engine();
        initialize_data();
        initialize_topography();
    }

    ~TrajectoryIntegrator() {
        if (engine_) gr_destroy(engine_);
    }

    std::unique_ptr<TrajectorySet> compute() {
        if (computed_)
            user_error("compute() was already called on this TrajectoryIntegrator; the loader has been consumed. "
                       "Create a new TrajectoryIntegrator for another run.");
        computed_ = true;
        const auto &ac = settings_.AdditionalCompute;
        if (ac.size() > GR_MAX_EXPRESSIONS) user_error("At most 4 AdditionalCompute expressions are supported.");
        const bool comp = !ac.empty();
        // variants the reference cannot pick (TrajectoryIntegrator.gen.py:52-53, 184-187)
        if (!comp && settings_.ConstantsMode != ConstantsMode::Off)
            user_error("No kernel could be picked for your settings configuration.");
        if (space_ == granite::Space::Space2D && (settings_.CurvatureMode == CurvatureMode::TotalCurvature ||
                                                  settings_.CurvatureMode == CurvatureMode::IndividualAndTotalCurvature))
            user_error("No kernel could be picked for your settings configuration.");
        std::vector<const char *> vn, cn;
        for (auto &k : vol_keys_) vn.push_back(k.c_str());
        for (auto &k : con_keys_) cn.push_back(k.c_str());
        for (size_t i = 0; i < ac.size(); ++i)
            check(gr_compile_expression(engine_, static_cast<int32_t>(i), ac[i].c_str(), vn.data(),
                                        static_cast<int32_t>(vn.size()), cn.data(), static_cast<int32_t>(cn.size())));
        pending_ = nullptr;
        const int rc = gr_run(engine_, &TrajectoryIntegrator::loader_cb, this);
        if (pending_) std::rethrow_exception(pending_);
        check(rc);
        return collect(comp);
    }

  private:
    IntegratorSettings settings_;
    DataLoader &loader_;
    granite::Space space_{granite::Space::Space3D};
    size_t n_{0};
    int dim_{3};
    std::vector<float> seeds_;
    gr_engine *engine_{nullptr};
    std::vector<std::string> vol_keys_, con_keys_;
    std::exception_ptr pending_;
    bool computed_{false};

    static void check(int rc) {
        if (rc != GR_OK) throw std::runtime_error(gr_last_error());
    }

    bool dyn_any() const {
        return settings_.WindfieldMode == WindfieldMode::Dynamic || settings_.UpLiftMode == UpLiftMode::Dynamic ||
               settings_.AdditionalVolumeMode == AdditionalVolumeMode::Dynamic ||
               settings_.ConstantsMode == ConstantsMode::Dynamic;
    }

    void create_engine() {
        gr_settings s;
        gr_settings_default(&s);
        const auto &S = settings_;
        s.space = static_cast<int32_t>(S.Space);
        s.integrator = static_cast<int32_t>(S.Integrator);
        s.windfield_mode = static_cast<int32_t>(S.WindfieldMode);
        s.constants_mode = static_cast<int32_t>(S.ConstantsMode);
        s.volume_mode = static_cast<int32_t>(S.AdditionalVolumeMode);
        s.uplift_mode = static_cast<int32_t>(S.UpLiftMode);
        s.border_mode = static_cast<int32_t>(S.BorderMode);
        s.curvature_mode = static_cast<int32_t>(S.CurvatureMode);
        s.abort_mode = static_cast<int32_t>(S.AbortMode);
        s.reverse = S.Reverse ? 1 : 0;
        s.minimum_alive = S.MinimumAliveParticles;
        if (S.GridScale.empty() || S.GridScale.size() > 3) user_error("Invalid GridScale dimension.");
        s.grid_scale_len = static_cast<int32_t>(S.GridScale.size());
        for (size_t k = 0; k < S.GridScale.size(); ++k) s.grid_scale[k] = S.GridScale[k];
        s.offset_len = static_cast<int32_t>(std::min<size_t>(S.Offset.size(), 3));
        for (size_t k = 0; k < S.Offset.size() && k < 3; ++k) s.offset[k] = S.Offset[k];
        s.sphere_radius = S.SphereRadius;
        s.delta_t = S.DeltaT;
        s.data_time_distance = S.DataTimeDistance;
        s.maximum_length = S.MaximumLength;
        s.maximum_simulation_time = S.MaximumSimulationTime;
        s.save_interval = static_cast<int64_t>(S.SaveInterval);
        s.storage = static_cast<int32_t>(S.WindStorage);
        s.time_mode = S.Float64Time ? 1 : 0;
        s.compensated = S.CompensatedPositions ? 1 : 0;
        s.ring_slots = S.RingSlots;
        s.steps_per_launch = S.StepsPerLaunch;
        s.sort_interval = S.SortInterval;
        s.block_size = S.BlockSize;
        s.device = S.Device;
        s.layout = S.WindLayout;
        s.filter_weights = S.ReferenceFilter ? 1 : 0;
        check(gr_create(&s, &engine_));
        check(gr_set_seeds(engine_, seeds_.data(), static_cast<int64_t>(n_), dim_));
    }

    void load_windfield(int64_t snapshot) {
        std::vector<py::array_t<float>> wf = loader_.windfield();
        if (static_cast<int>(wf.size()) < dim_)
            user_error(dim_ == 3 ? "Invalid dataset was provided. Wrong amout of data (3D)."
                                 : "Invalid dataset was provided. Wrong amout of data (2D).");
        std::vector<farray> planes;
        std::vector<const float *> ptr;
        for (int c = 0; c < dim_; ++c) {
            planes.push_back(farray::ensure(wf[c]));
            if (!planes.back() || planes.back().ndim() != dim_)
                user_error(dim_ == 3 ? "Invalid dataset was provided. Wrong amout of data (3D)."
                                     : "Invalid dataset was provided. Wrong amout of data (2D).");
            ptr.push_back(planes.back().data());
        }
        const auto &p = planes[0];
        const int64_t nz = dim_ == 3 ? p.shape(0) : 1, ny = p.shape(dim_ - 2), nx = p.shape(dim_ - 1);
        for (int c = 1; c < dim_; ++c)
            for (int d = 0; d < dim_; ++d)
                if (planes[c].shape(d) != p.shape(d))
                    user_error(dim_ == 3 ? "Invalid dataset was provided. Shape does not match in x dimension (3D)."
                                         : "Invalid dataset was provided. Shape does not match in x dimension (2D).");
        check(gr_load_windfield(engine_, snapshot, ptr.data(), dim_, nz, ny, nx));
        nz_ = nz; ny_ = ny; nx_ = nx;
    }

    void load_volumes(int64_t snapshot, bool first) {
        py::object obj = py::cast(loader_).attr("additionalVolumes")();
        map_t m = obj.cast<map_t>();
        if (first && m.size() > GR_MAX_VOLUMES) user_warning("You provided more additional volumes than supported.");
        for (auto &kv : ordered(m, obj)) {
            int idx = -1;
            for (size_t k = 0; k < vol_keys_.size(); ++k)
                if (vol_keys_[k] == kv.first) idx = static_cast<int>(k);
            if (first && idx < 0) {
                if (vol_keys_.size() == GR_MAX_VOLUMES) break;
                vol_keys_.push_back(kv.first);
                idx = static_cast<int>(vol_keys_.size()) - 1;
            }
            if (idx < 0) continue;   // keys unknown at construction are skipped (cpp:280)
            const farray &a = kv.second;
            if (a.ndim() != dim_)
                user_error(dim_ == 3 ? "Invalid dataset was provided. Wrong amout of data (3D)."
                                     : "Invalid dataset was provided. Wrong amout of data (2D).");
            const int64_t nz = dim_ == 3 ? a.shape(0) : 1, ny = a.shape(dim_ - 2), nx = a.shape(dim_ - 1);
            check(gr_load_volume(engine_, snapshot, idx, a.data(), nz, ny, nx));
        }
    }

    void load_constants(int64_t snapshot, bool first) {
        py::object obj = py::cast(loader_).attr("constants")();
        map_t m = obj.cast<map_t>();
        if (m.size() > GR_MAX_CONSTANTS) user_warning("You provided more constants than supported.");
        for (auto &kv : ordered(m, obj)) {
            int idx = -1;
            for (size_t k = 0; k < con_keys_.size(); ++k)
                if (con_keys_[k] == kv.first) idx = static_cast<int>(k);
            if (first && idx < 0) {
                if (con_keys_.size() == GR_MAX_CONSTANTS) break;
                con_keys_.push_back(kv.first);
                idx = static_cast<int>(con_keys_.size()) - 1;
            }
            if (idx < 0) continue;
            const farray &a = kv.second;
            if (static_cast<size_t>(a.size()) < n_) user_error("Constant dimension does not match number of particles.");
            check(gr_load_constant(engine_, snapshot, idx, a.data(), static_cast<int64_t>(n_)));
        }
    }

    void load_uplift(int64_t snapshot) {
        farray a = farray::ensure(loader_.uplift());
        if (!a || a.ndim() < 1 || static_cast<size_t>(a.shape(0)) != n_)
            user_error("Uplift dimension does not match number of particles.");
        if (static_cast<size_t>(a.size()) < n_ * dim_) user_error("Uplift dimension does not match number of particles.");
        check(gr_load_uplift(engine_, snapshot, a.data(), static_cast<int64_t>(n_), dim_));
    }

    // initializeData (cpp:146-259)
    void initialize_data() {
        load_windfield(0);
        if (settings_.AdditionalVolumeMode != AdditionalVolumeMode::Off) load_volumes(0, true);
        if (settings_.ConstantsMode != ConstantsMode::Off) load_constants(0, true);
        if (settings_.UpLiftMode != UpLiftMode::Off) load_uplift(0);
        if (dyn_any()) {
            if (loader_.step()) update_data(1);
            else user_error("Cannot increment loader.");
        }
    }

    // updateData (cpp:261-360)
    void update_data(int64_t snapshot) {
        if (settings_.WindfieldMode == WindfieldMode::Dynamic) load_windfield(snapshot);
        if (settings_.AdditionalVolumeMode == AdditionalVolumeMode::Dynamic) load_volumes(snapshot, false);
        if (settings_.ConstantsMode == ConstantsMode::Dynamic) load_constants(snapshot, false);
        if (settings_.UpLiftMode == UpLiftMode::Dynamic) load_uplift(snapshot);
    }

    // initializeTopography (cpp:635-663)
    void initialize_topography() {
        if (settings_.Topography.size() > 0) {
            farray t = farray::ensure(settings_.Topography);
            if (t.ndim() != 2) user_error("Invalid topography was provided. Wrong dimension of data (2D).");
            if (t.shape(1) != nx_ || t.shape(0) != ny_) user_error("Topography dimensions does not match to provided data!");
            check(gr_set_topography(engine_, t.data(), t.shape(0), t.shape(1)));
        }
    }

    static int loader_cb(void *user, gr_engine *, int64_t snapshot) {
        auto *self = static_cast<TrajectoryIntegrator *>(user);
        try {
            if (!self->loader_.step()) return 0;
            self->update_data(snapshot);
            return 1;
        } catch (...) {
            self->pending_ = std::current_exception();
            return -1;
        }
    }

    // Result storage: page-locked (one DMA per result) with PinnedResults, else plain numpy.
    py::array_t<float> result_array(const std::vector<py::ssize_t> &shape) const {
        return settings_.PinnedResults ? pinned_empty(shape) : py::array_t<float>(shape);
    }

    // Results are fetched after the run.  Streaming them out during the run
    // (gr_set_result_destinations) does not pay here: the run is bound by the snapshot uploads
    // over the same link, and both directions together moved less than one after the other.
    std::unique_ptr<TrajectorySet> collect(bool comp) {
        gr_result_info info;
        check(gr_result_info_get(engine_, &info));
        auto set = std::make_unique<TrajectorySet>();
        set->space = space_;
        set->n = n_;
        set->dim = static_cast<size_t>(dim_);
        set->particle_steps = info.particle_steps;
        const auto N = static_cast<py::ssize_t>(n_);
        set->traj = result_array({N, static_cast<py::ssize_t>(info.records), static_cast<py::ssize_t>(dim_)});
        check(gr_fetch_positions(engine_, set->traj.mutable_data(), static_cast<int64_t>(set->traj.size())));
        std::vector<int32_t> st(n_);
        check(gr_fetch_status(engine_, st.data(), static_cast<int64_t>(n_)));
        set->abort_reasons.resize(n_);
        for (size_t i = 0; i < n_; ++i) set->abort_reasons[i] = static_cast<AbortReason>(st[i]);
        if (settings_.AbortMode != AbortMode::Time) {
            set->lengths.resize(n_);
            check(gr_fetch_lengths(engine_, set->lengths.data(), static_cast<int64_t>(n_)));
        }
        if (settings_.CurvatureMode != CurvatureMode::Off) {
            set->total_curvature.resize(n_);
            check(gr_fetch_total_curvature(engine_, set->total_curvature.data(), static_cast<int64_t>(n_)));
        }
        set->curv = result_array({N, static_cast<py::ssize_t>(info.curvature_records)});
        if (info.curvature_records > 0)
            check(gr_fetch_curvatures(engine_, set->curv.mutable_data(), static_cast<int64_t>(set->curv.size())));
        if (settings_.AdditionalVolumeMode != AdditionalVolumeMode::Off) {
            for (size_t k = 0; k < vol_keys_.size(); ++k) {
                py::array_t<float> a = result_array({N, static_cast<py::ssize_t>(info.info_records)});
                check(gr_fetch_volume_info(engine_, static_cast<int32_t>(k), a.mutable_data(), static_cast<int64_t>(a.size())));
                set->volume_data.emplace_back(vol_keys_[k], a);
            }
        }
        if (comp) {
            set->num_compute = settings_.AdditionalCompute.size();
            for (size_t e = 0; e < set->num_compute; ++e) {
                py::array_t<float> a = result_array({N, static_cast<py::ssize_t>(info.info_records)});
                check(gr_fetch_compute_info(engine_, static_cast<int32_t>(e), a.mutable_data(), static_cast<int64_t>(a.size())));
                set->compute_data.push_back(a);
            }
        }
        return set;
    }

    int64_t nz_{0}, ny_{0}, nx_{0};
};

}  // namespace granite

PYBIND11_MODULE(_pygranite, m) {
    using namespace granite;
    m.doc() = "B200-native drop-in for pygranite: trajectory integration of particles through "
              "time-dependent 2D/3D wind fields on NVIDIA B200 GPUs.";

    // registration order as source/pygranite.cpp:41-100 (module-level names: last one wins)
    py::enum_<Space>(m, "Space").value("Space2D", Space::Space2D).value("Space3D", Space::Space3D).export_values();
    py::enum_<Integrator>(m, "Integrator")
        .value("ExplicitEuler", Integrator::ExplicitEuler)
        .value("ClassicRungeKutta", Integrator::ClassicRungeKutta)
        .export_values();
    py::enum_<AbortReason>(m, "AbortReason")
        .value("Time", AbortReason::Time)
        .value("Domain", AbortReason::Domain)
        .value("Length", AbortReason::Length)
        .value("Topography", AbortReason::Topography)
        .value("Wind", AbortReason::Wind)
        .export_values();
    py::enum_<BorderMode>(m, "BorderMode")
        .value("Block", BorderMode::Block)
        .value("LoopX", BorderMode::LoopX)
        .value("LoopY", BorderMode::LoopY)
        .value("LoopXY", BorderMode::LoopXY)
        .export_values();
    py::enum_<CurvatureMode>(m, "CurvatureMode")
        .value("Off", CurvatureMode::Off)
        .value("FastTotalCurvature", CurvatureMode::FastTotalCurvature)
        .value("IndividualAndTotalCurvature", CurvatureMode::IndividualAndTotalCurvature)
        .value("TotalCurvature", CurvatureMode::TotalCurvature)
        .export_values();
    py::enum_<AbortMode>(m, "AbortMode")
        .value("Time", AbortMode::Time)
        .value("Length", AbortMode::Length)
        .value("FitLength", AbortMode::FitLength)
        .export_values();
    py::enum_<UpLiftMode>(m, "UpLiftMode")
        .value("Off", UpLiftMode::Off)
        .value("Constant", UpLiftMode::Constant)
        .value("Dynamic", UpLiftMode::Dynamic)
        .export_values();
    py::enum_<WindfieldMode>(m, "WindfieldMode")
        .value("Constant", WindfieldMode::Constant)
        .value("Dynamic", WindfieldMode::Dynamic)
        .export_values();
    py::enum_<AdditionalVolumeMode>(m, "AdditionalVolumeMode")
        .value("Off", AdditionalVolumeMode::Off)
        .value("Constant", AdditionalVolumeMode::Constant)
        .value("Dynamic", AdditionalVolumeMode::Dynamic)
        .export_values();
    py::enum_<ConstantsMode>(m, "ConstantsMode")
        .value("Off", ConstantsMode::Off)
        .value("Constant", ConstantsMode::Constant)
        .value("Dynamic", ConstantsMode::Dynamic)
        .export_values();
    // engine extension (not in the reference)
    py::enum_<WindStorage>(m, "WindStorage")
        .value("Float32", WindStorage::Float32)
        .value("BFloat16", WindStorage::BFloat16)
        .value("Float16", WindStorage::Float16);

    py::class_<IntegratorSettings>(m, "IntegratorSettings")
        .def(py::init<>())
        .def_readwrite("Space", &IntegratorSettings::Space)
        .def_readwrite("Integrator", &IntegratorSettings::Integrator)
        .def_readwrite("DeltaT", &IntegratorSettings::DeltaT)
        .def_readwrite("SaveInterval", &IntegratorSettings::SaveInterval)
        .def_readwrite("MinimumAliveParticles", &IntegratorSettings::MinimumAliveParticles)
        .def_readwrite("GridScale", &IntegratorSettings::GridScale)
        .def_readwrite("DataTimeDistance", &IntegratorSettings::DataTimeDistance)
        .def_readwrite("Topography", &IntegratorSettings::Topography)
        .def_readwrite("MaximumLength", &IntegratorSettings::MaximumLength)
        .def_readwrite("AdditionalCompute", &IntegratorSettings::AdditionalCompute)
        .def_readwrite("Offset", &IntegratorSettings::Offset)
        .def_readwrite("Reverse", &IntegratorSettings::Reverse)
        .def_readwrite("SphereRadius", &IntegratorSettings::SphereRadius)
        .def_readwrite("BorderMode", &IntegratorSettings::BorderMode)
        .def_readwrite("CurvatureMode", &IntegratorSettings::CurvatureMode)
        .def_readwrite("AbortMode", &IntegratorSettings::AbortMode)
        .def_readwrite("UpLiftMode", &IntegratorSettings::UpLiftMode)
        .def_readwrite("WindfieldMode", &IntegratorSettings::WindfieldMode)
        .def_readwrite("AdditionalVolumeMode", &IntegratorSettings::AdditionalVolumeMode)
        .def_readwrite("ConstantsMode", &IntegratorSettings::ConstantsMode)
        .def_readwrite("MaximumSimulationTime", &IntegratorSettings::MaximumSimulationTime)
        .def_readwrite("WindStorage", &IntegratorSettings::WindStorage)
        .def_readwrite("Float64Time", &IntegratorSettings::Float64Time)
        .def_readwrite("CompensatedPositions", &IntegratorSettings::CompensatedPositions)
        .def_readwrite("RingSlots", &IntegratorSettings::RingSlots)
        .def_readwrite("StepsPerLaunch", &IntegratorSettings::StepsPerLaunch)
        .def_readwrite("SortInterval", &IntegratorSettings::SortInterval)
        .def_readwrite("BlockSize", &IntegratorSettings::BlockSize)
        .def_readwrite("Device", &IntegratorSettings::Device)
        .def_readwrite("WindLayout", &IntegratorSettings::WindLayout)
        .def_readwrite("PinnedResults", &IntegratorSettings::PinnedResults)
        .def_readwrite("ReferenceFilter", &IntegratorSettings::ReferenceFilter);

    m.def("pinned_empty", &pinned_empty, py::arg("shape"),
          "Uninitialised float32 array in page-locked host memory (engine extension).  Loader data "
          "and results in such arrays move by one DMA, without staging copies.");

    py::class_<TrajectoryIntegrator>(m, "TrajectoryIntegrator")
        .def(py::init<IntegratorSettings &, DataLoader &, TrajectorySet &>(), py::keep_alive<1, 3>())
        .def("compute", &TrajectoryIntegrator::compute);

    py::class_<DataLoader, PyDataLoader>(m, "DataLoader")
        .def(py::init<>())
        .def("step", &DataLoader::step)
        .def("windfield", &DataLoader::windfield)
        .def("uplift", &DataLoader::uplift)
        .def("constants", &DataLoader::constants)
        .def("additionalVolumes", &DataLoader::additionalVolumes);

    py::class_<TrajectorySet>(m, "TrajectorySet")
        .def(py::init<py::array_t<float>>())
        .def("trajectory", &TrajectorySet::trajectory)
        .def("trajectories", &TrajectorySet::trajectories)
        .def("cloud", &TrajectorySet::cloud)
        .def("totalCurvatures", &TrajectorySet::totalCurvatures)
        .def("curvatures", &TrajectorySet::curvatures)
        .def("individualLengths", &TrajectorySet::individualLengths)
        .def("volumeInfo", &TrajectorySet::volumeInfo)
        .def("computeInfo", &TrajectorySet::computeInfo)
        .def("lengthTrajectories", &TrajectorySet::lengthTrajectories)
        .def("abortReasons", &TrajectorySet::abortReasons)
        .def("numberTrajectories", &TrajectorySet::numberTrajectories)
        // not in the reference: alive particles advanced by the run that produced this set,
        // summed over its steps (0 for a set made from seeds)
        .def("particleSteps", [](const TrajectorySet &t) { return t.particle_steps; });
}
