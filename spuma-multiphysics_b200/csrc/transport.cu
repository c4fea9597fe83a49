// reactive_transport_* C ABI on B200: host object, residency/version contract,
// and launch sequencing for the face-graph and structured Cartesian kernels.
//
// The contract (argument meaning, validation messages, return codes 0/1/2/-1,
// version tokens, RK stage rules, residency invalidation on failure) follows
// src/reactiveTransport/reactiveTransport.cpp:381-1815 and
// src/reactiveTransport/reactiveTransport.h:48-141. Execution is CUDA only:
// backend 0 (the reference's serial CPU loop) is rejected, never emulated.
#include "cartesian_kernels.cuh"
#include "capillary_resident.cuh"
#include "wale_pr.cuh"
#include <cub/device/device_radix_sort.cuh>
#include "../../include/reactive_b200_transport.h"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

namespace rb200 {
namespace {

size_t product(size_t a, size_t b) {
    require(!b || a <= std::numeric_limits<size_t>::max() / b, "Transport allocation size overflow");
    return a * b;
}

struct DeviceArena {
    std::vector<void*> blocks;
    uint64_t bytes = 0, peak = 0;
    double limit = 0;
    template <class T> T* get(size_t n) {
        if (!n) return nullptr;
        const size_t b = product(n, sizeof(T));
        require(double(bytes) + double(b) <= limit, "Transport exceeds maxDeviceMemoryGB/workspace budget");
        void* p = nullptr;
        check(cudaMalloc(&p, b), "cudaMalloc");
        blocks.push_back(p);
        bytes += b;
        peak = std::max(peak, bytes);
        return static_cast<T*>(p);
    }
    ~DeviceArena() { for (void* p : blocks) cudaFree(p); }
};

// One thread per cell: the phase-aware cp and effective species enthalpies of
// the accepted states (wale_pr.cuh); the first failing cell (lowest index) and
// its status go to `failure` as (cell << 8) | status.
__global__ void walePrProperties(const ReactiveB200HemModel* model, const double* q,
                                 const ReactiveThermoState* states, const double* color, const double* curvature,
                                 double sigma, size_t cells, size_t species, double* h, double* cp,
                                 unsigned long long* failure, bool enthalpies) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < cells; c += size_t(blockDim.x) * gridDim.x) {
        double local[mix::kMaxNs] = {};
        double candidate = 0;
        const int status = walepr::properties(*model, enthalpies ? q + c * species : nullptr, states[c], color[c],
                                              sigma * curvature[c], local, candidate, enthalpies);
        if (status != walepr::SUCCESS) {
            atomicMin(failure, ((unsigned long long)c << 8) | unsigned(status));
            continue;
        }
        cp[c] = candidate;
        if (enthalpies)
            for (size_t k = 0; k < species; ++k) h[c * species + k] = local[k];
    }
}

// Publishes a successful property build into the WALE scalar fields.
__global__ void walePrCommit(size_t cells, size_t species, size_t stride, const double* sourceH,
                             const double* sourceCp, double* destinationH, double* destinationCp, bool enthalpies,
                             bool heatFlux) {
    for (size_t c = blockIdx.x * size_t(blockDim.x) + threadIdx.x; c < cells; c += size_t(blockDim.x) * gridDim.x) {
        if (heatFlux) destinationCp[c] = sourceCp[c];
        if (enthalpies)
            for (size_t k = 0; k < species; ++k) destinationH[k * stride + c] = sourceH[c * species + k];
    }
}

struct Transport {
    std::mutex entry;
    int device = 0;
    cudaStream_t stream = nullptr;
    ReactiveTransportConfig cfg{};
    GraphView v{};
    DeviceArena arena;
    double* q = nullptr;        // SoA nv x all (the resident RK input)
    double* initial = nullptr;  // SoA nv x all (the other RK buffer)
    double* rhs = nullptr;      // SoA nv x cells (materialised diagnostic)
    double* staging = nullptr;  // cell-major bridge, max(cells, fixed) x max(nv, 9... )
    size_t stagingDoubles = 0;
    double* reduceScratch = nullptr;
    size_t reduceBlocks = 0;
    double* boundaryRate = nullptr;
    ReactiveTransportState* stateDevice = nullptr;
    unsigned* flags = nullptr;  // [0] WALE failure
    unsigned long long* invalid = nullptr;  // first invalid uploaded state / primitive
    // structured Cartesian fast path (device-resident entries only)
    bool boxDetected = false, structured = false;
    CartView box{};
    bool mixed = false;
    float* gradF = nullptr;  // 9 x cells, mixed path
    float* nutF = nullptr;   // cells, mixed path
    double* ledgerPartial = nullptr;
    unsigned ledgerBlocks = 0;
    ReactiveTransportStats stats{};
    ReactiveTransportProfile profile{};
    ReactiveTransportDeviceProfile deviceProfile{};
    ReactiveTransportProfileV21 cost{};
    ReactiveWaleProfileV1 waleProfile{1, sizeof(ReactiveWaleProfileV1), 0, 0, 0, 0};
    ReactiveWaleScalarProfileV1 waleScalarProfile{1, sizeof(ReactiveWaleScalarProfileV1), 0, 0, 0};
    bool scalarCp = false, scalarH = false;  // WALE scalar fields present for the next stage
    // diffuse capillary closure: the published geometry and the host copies of
    // its inputs and outputs that let an identical request skip the device
    ReactiveCapillaryProfileV1 capillaryProfile{1, sizeof(ReactiveCapillaryProfileV1), 0, 0, 0, 0, 0, 0, 0};
    bool colorReady = false, geometryShadowValid = false;
    std::vector<double> colorShadow, fixedColorShadow, energyShadow, curvatureShadow;
    uint64_t geometryBuildsSkipped = 0;
    double* colorDevice = nullptr;  // cells + fixed
    // the resident capillary closure's device buffers (allocated by its first begin)
    struct CapillaryResident {
        size_t cells = 0, species = 0, sortBytes = 0;
        double sigma = 0;
        int equilibrium = 1;
        bool ready = false;
        double *q = nullptr, *bulk = nullptr, *energy = nullptr, *color = nullptr, *jump = nullptr;
        double *colorBefore = nullptr, *jumpBefore = nullptr, *energyBefore = nullptr;
        double *flashedColor = nullptr, *flashedJump = nullptr, *flashedEnergy = nullptr;
        ReactiveThermoState* seed = nullptr;
        ReactiveGpuHemOutputV1* output = nullptr;
        ReactiveGpuHemCapillaryInputV2* capillary = nullptr;
        uint16_t *keys = nullptr, *sortedKeys = nullptr;
        uint32_t *cells32 = nullptr, *order = nullptr;
        void* sortTemp = nullptr;
        unsigned long long* scalars = nullptr;  // [0] dirty count, [1] residual bits
        unsigned* flags = nullptr;
        std::vector<double> fixedColor;
    } resident;
    // the WALE PR scalar-property pass (src/reactiveTransport/reactiveTransport.cpp:703-828)
    bool walePrInstalled = false, walePrReady = false, walePrStatesCurrent = false;
    ReactiveWalePrEpochV1 walePrEpoch{};
    uint64_t walePrLastThermoVersion = 0;
    ReactiveWalePrProfileV1 walePrProfile{1, sizeof(ReactiveWalePrProfileV1), 0, 0, 0, 0, 0, 0, 0.0};
    ReactiveB200HemModel* walePrModel = nullptr;
    ReactiveThermoState* walePrStates = nullptr;
    double *walePrQ = nullptr, *walePrH = nullptr, *walePrCp = nullptr;
    unsigned long long* walePrFailure = nullptr;
    std::vector<double> walePrHostQ;
    std::string physicalHash;
    uint64_t attemptId = 0, lastAttempt = 0, tokenStage = 0;
    bool attemptOpen = false;
    uint64_t residentVersion = 0, highestVersion = 0;
    bool haveResident = false, haveInitial = false;
    double stageDt = 0;
    uint64_t deviceCopies = 0, synchronizations = 0, memcpyCalls = 0;
    char error[1024] = {0};

    Transport(int backend, const ReactiveTransportConfig& c, const double* volumes,
              const ReactiveTransportFace* faces, const double* fixedQ, const ReactiveTransportState* fixedStates,
              const double* fixedY, const double* fixedH, const ReactiveTransportOptionsV2* options,
              const ReactiveTransportOptionsV21* options21) {
        require(backend == 0 || backend == 1, "Unknown transport backend");
        require(backend == 1, "This library executes on CUDA only; backend 0 (serial CPU) is not provided");
        int count = 0;
        check(cudaGetDeviceCount(&count), "cudaGetDeviceCount");
        require(count > 0, "No CUDA device");
        check(cudaGetDevice(&device), "cudaGetDevice");
        check(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
        cfg = c;
        arena.limit = cfg.maxBytes;
        if (options) {
            require(options->abiVersion == 1 && options->structBytes == sizeof(*options) && options->bridgeCells > 0,
                    "Invalid transport options ABI");
            require(options->physicalModelHash[64] == 0 && std::strlen(options->physicalModelHash) == 64,
                    "Invalid transport model hash");
            physicalHash = options->physicalModelHash;
            require(!options->recomputeGas, "Generated NASA gas properties are not part of this build");
        }
        if (options21) cost.blockThreads = options21->blockThreads;
        cost.slots = 1;
        require(cfg.cells && cfg.species && cfg.faces, "Empty transport mesh/model");
        require(cfg.cells <= size_t(INT64_MAX) && cfg.faces < size_t(INT64_MAX) && cfg.fixed <= size_t(INT64_MAX),
                "Transport index overflow");
        require(cfg.mechanical ? cfg.variables == cfg.species + 6
                               : (cfg.variables >= cfg.species + 4 && cfg.variables <= cfg.species + 6),
                "Wrong transport conserved-variable count");
        require(std::isfinite(cfg.maxBytes) && cfg.maxBytes > 0, "Invalid transport memory budget");
        require(std::isfinite(cfg.waveFactor) && cfg.waveFactor >= 1, "Invalid transport wave factor");
        require(std::isfinite(cfg.viscosity) && std::isfinite(cfg.conductivity) && std::isfinite(cfg.diffusivity)
                    && cfg.viscosity >= 0 && cfg.conductivity >= 0 && cfg.diffusivity >= 0,
                "Invalid transport coefficients");
        require(!cfg.mechanical || (cfg.viscosity == 0 && cfg.conductivity == 0 && cfg.diffusivity == 0),
                "Mechanical transport requires inviscid, non-diffusive model");
        require(volumes && faces, "Null transport geometry");
        require(cfg.cells <= std::numeric_limits<size_t>::max() - cfg.fixed, "Fixed-state index overflow");
        const size_t all = cfg.cells + cfg.fixed;
        std::vector<int64_t> row(cfg.cells + 1, 0), boundary;
        for (size_t i = 0; i < cfg.cells; ++i)
            require(std::isfinite(volumes[i]) && volumes[i] > 0, "Invalid transport volume");
        for (size_t i = 0; i < cfg.faces; ++i) {
            const auto& f = faces[i];
            require(f.owner >= 0 && size_t(f.owner) < cfg.cells && f.neighbour >= -1
                        && (f.neighbour < 0 || size_t(f.neighbour) < cfg.cells),
                    "Invalid transport face cell");
            require(f.kind >= 0 && f.kind <= 3 && (f.kind == 0) == (f.neighbour >= 0), "Invalid transport face kind");
            require(f.kind != 3 || (f.fixed >= 0 && size_t(f.fixed) < cfg.fixed && !cfg.mechanical),
                    "Invalid fixed boundary state index");
            double norm = 0;
            for (double x : f.normal) norm += x * x;
            require(std::isfinite(norm) && std::abs(norm - 1) < 1e-8, "Invalid transport unit normal");
            require(std::isfinite(f.area) && std::isfinite(f.distance) && std::isfinite(f.ownerWeight) && f.area > 0
                        && f.distance > 0 && f.ownerWeight >= 0 && f.ownerWeight <= 1,
                    "Invalid transport face geometry");
            ++row[f.owner + 1];
            if (f.neighbour >= 0) ++row[f.neighbour + 1];
            else boundary.push_back(int64_t(i));
        }
        for (size_t i = 0; i < cfg.cells; ++i) row[i + 1] += row[i];
        std::vector<int64_t> incidence(size_t(row.back()));
        auto next = row;
        for (size_t i = 0; i < cfg.faces; ++i) {
            incidence[size_t(next[faces[i].owner]++)] = -int64_t(i) - 1;
            if (faces[i].neighbour >= 0) incidence[size_t(next[faces[i].neighbour]++)] = int64_t(i) + 1;
        }
        std::vector<double> inverse(cfg.cells);
        for (size_t i = 0; i < cfg.cells; ++i) {
            inverse[i] = 1 / volumes[i];
            require(std::isfinite(inverse[i]), "Invalid inverse volume");
        }
        validateStates(fixedStates, cfg.fixed);
        std::vector<ReactiveTransportPrimitive> fixedPrimitive(cfg.fixed);
        for (size_t i = 0; i < cfg.fixed; ++i) {
            auto& p = fixedPrimitive[i];
            for (size_t k = 0; k < cfg.species; ++k) p.rho += fixedQ[i * cfg.variables + k];
            require(std::isfinite(p.rho) && p.rho > 0, "Invalid fixed density");
            for (int d = 0; d < 3; ++d) {
                p.u[d] = fixedQ[i * cfg.variables + cfg.species + d] / p.rho;
                require(std::isfinite(p.u[d]), "Invalid fixed velocity");
            }
        }
        auto* faceDevice = arena.get<ReactiveTransportFace>(cfg.faces);
        auto* rowDevice = arena.get<int64_t>(row.size());
        auto* incidenceDevice = arena.get<int64_t>(incidence.size());
        auto* boundaryDevice = arena.get<int64_t>(boundary.size());
        auto* invDevice = arena.get<double>(cfg.cells);
        stateDevice = arena.get<ReactiveTransportState>(all);
        q = arena.get<double>(product(all, cfg.variables));
        initial = arena.get<double>(product(all, cfg.variables));
        auto* primitive = arena.get<ReactiveTransportPrimitive>(all);
        auto* work = arena.get<double>(product(cfg.faces, FW_FIELDS));
        auto* carrier = arena.get<int>(cfg.faces);
        auto* faceSpeed = arena.get<double>(cfg.faces);
        auto* step = arena.get<double>(cfg.cells);
        boundaryRate = arena.get<double>(cfg.variables);
        flags = arena.get<unsigned>(4);
        invalid = arena.get<unsigned long long>(2);
        reduceBlocks = std::min<size_t>(1024, (cfg.cells + 255) / 256);
        reduceScratch = arena.get<double>(reduceBlocks + 1);
        double* gasY = nullptr;
        double* gasH = nullptr;
        if (cfg.diffusivity > 0) {
            gasY = arena.get<double>(product(all, cfg.species));
            gasH = arena.get<double>(product(all, cfg.species));
        }
        double* grad = cfg.viscosity > 0 ? arena.get<double>(product(cfg.cells, 9)) : nullptr;
        stagingDoubles = std::max(product(std::max(cfg.cells, cfg.fixed), cfg.variables),
                                  product(std::max(cfg.cells, cfg.fixed), cfg.species));
        staging = arena.get<double>(stagingDoubles);
        deviceProfile.faceWorkspaceBytes = product(cfg.faces, FW_FIELDS * sizeof(double) + sizeof(int) + sizeof(double));
        profile.boundaryPartitions = 1;

        upload(faceDevice, faces, cfg.faces);
        upload(rowDevice, row.data(), row.size());
        upload(incidenceDevice, incidence.data(), incidence.size());
        upload(boundaryDevice, boundary.data(), boundary.size());
        upload(invDevice, inverse.data(), cfg.cells);
        upload(stateDevice + cfg.cells, fixedStates, cfg.fixed);
        upload(primitive + cfg.cells, fixedPrimitive.data(), cfg.fixed);
        check(cudaMemsetAsync(flags, 0, 4 * sizeof(unsigned), stream), "cudaMemsetAsync");

        v.cells = cfg.cells; v.fixed = cfg.fixed; v.all = all; v.ns = cfg.species; v.nv = cfg.variables;
        v.faces = cfg.faces; v.nBoundary = boundary.size(); v.mechanical = cfg.mechanical;
        v.viscosity = cfg.viscosity; v.conductivity = cfg.conductivity; v.diffusivity = cfg.diffusivity;
        v.waveFactor = cfg.waveFactor;
        v.face = faceDevice; v.row = rowDevice; v.incidence = incidenceDevice; v.boundary = boundaryDevice;
        v.invV = invDevice; v.state = stateDevice; v.q = q; v.primitive = primitive; v.grad = grad;
        v.gasY = gasY; v.gasH = gasH; v.work = work; v.carrier = carrier; v.faceSpeed = faceSpeed; v.step = step;
        v.waleError = flags;
        boxDetected = detectBox(faces, cfg.faces - boundary.size(), invDevice, primitive);
        structured = boxDetected;
        if (boxDetected) {
            ledgerBlocks = unsigned(std::min<size_t>(296, (box.nBoundary + 255) / 256));
            ledgerPartial = arena.get<double>(product(ledgerBlocks, cfg.variables));
        }

        packInto(q, fixedQ, cfg.fixed, cfg.variables, all, cfg.cells);
        packInto(initial, fixedQ, cfg.fixed, cfg.variables, all, cfg.cells);
        if (cfg.diffusivity > 0) {
            packInto(gasY, fixedY, cfg.fixed, cfg.species, all, cfg.cells);
            packInto(gasH, fixedH, cfg.fixed, cfg.species, all, cfg.cells);
        }
        finish();
    }
    ~Transport() {
        if (stream) { cudaStreamSynchronize(stream); cudaStreamDestroy(stream); }
    }

    // ---------------------------------------------------------------- transfers
    template <class T> void upload(T* dst, const T* src, size_t n) {
        if (!n) return;
        require(src && dst, "Null transport input buffer");
        check(cudaMemcpyAsync(dst, src, product(n, sizeof(T)), cudaMemcpyHostToDevice, stream), "H2D");
        stats.uploadedBytes += product(n, sizeof(T));
        ++memcpyCalls;
    }
    template <class T> void download(T* dst, const T* src, size_t n) {
        if (!n) return;
        require(src && dst, "Null transport output buffer");
        check(cudaMemcpyAsync(dst, src, product(n, sizeof(T)), cudaMemcpyDeviceToHost, stream), "D2H");
        stats.downloadedBytes += product(n, sizeof(T));
        ++memcpyCalls;
    }
    void finish() {
        ++synchronizations;
        check(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    }
    void launched() {
        check(cudaGetLastError(), "kernel launch");
        ++stats.kernelLaunches;
    }
    // Host cell-major rows -> SoA columns [offset, offset+count) of stride `stride`.
    void packInto(double* dst, const double* src, size_t count, size_t width, size_t stride, size_t offset) {
        if (!count) return;
        require(src, "Null packed source");
        upload(staging, src, count * width);
        packSoA<<<gridFor(count * width, 256), 256, 0, stream>>>(staging, dst, count, width, stride, offset);
        launched();
        ++cost.layoutLaunches;
        ++cost.layoutTiles;
    }
    void unpackFrom(double* dst, const double* src, size_t count, size_t width, size_t stride, size_t offset) {
        require(dst, "Null unpack output");
        unpackSoA<<<gridFor(count * width, 256), 256, 0, stream>>>(src, staging, count, width, stride, offset);
        launched();
        ++cost.layoutLaunches;
        ++cost.layoutTiles;
        download(dst, staging, count * width);
    }
    static void validateStates(const ReactiveTransportState* states, size_t count) {
        require(!count || states, "Null transport state");
        const size_t bad = firstFailure(count, [&](size_t c) {
            const auto& s = states[c];
            return std::isfinite(s.p) && s.p > 0 && std::isfinite(s.T) && s.T > 0 && std::isfinite(s.rho) && s.rho > 0
                && std::isfinite(s.sound) && s.sound > 0 && std::isfinite(s.cv) && s.cv > 0
                && std::isfinite(s.gasMass) && s.gasMass >= 0 && std::isfinite(s.dilatation);
        });
        require(bad == count, "Invalid recovered transport state");
    }
    void uploadQ(const double* hostQ) {
        packInto(q, hostQ, cfg.cells, cfg.variables, v.all, 0);
        ++profile.conservedUploads;
        profile.conservedUploadBytes += cfg.cells * cfg.variables * sizeof(double);
    }
    // States (and primitives) are validated on the device after the copy; the
    // call fails with the host validation's message before anything is formed
    // from them.
    void uploadState(const ReactiveTransportState* states, const ReactiveTransportPrimitive* primitive = nullptr) {
        require(!cfg.cells || states, "Null transport state");
        upload(stateDevice, states, cfg.cells);
        profile.stateUploadBytes += cfg.cells * sizeof(ReactiveTransportState);
        if (primitive) {
            upload(v.primitive, primitive, cfg.cells);
            profile.primitiveUploadBytes += cfg.cells * sizeof(ReactiveTransportPrimitive);
        }
        check(cudaMemsetAsync(invalid, 0xff, 2 * sizeof(unsigned long long), stream), "memset");
        validateUploads<<<gridFor(cfg.cells, 256), 256, 0, stream>>>(stateDevice, primitive ? v.primitive : nullptr,
                                                                    cfg.cells, invalid);
        launched();
        unsigned long long first[2];
        download(first, invalid, 2);
        finish();
        if (primitive && first[1] != ~0ull)
            require(false, (first[1] & 1) ? "Invalid primitive velocity" : "Invalid primitive density");
        require(first[0] == ~0ull, "Invalid recovered transport state");
    }
    void unpackQ(double* hostQ) {
        unpackFrom(hostQ, q, cfg.cells, cfg.variables, v.all, 0);
        profile.conservedDownloadBytes += cfg.cells * cfg.variables * sizeof(double);
    }

    // ---------------------------------------------------------------- kernels
    void launchPrimitives(const double* qSoA, cudaStream_t s) {
        GraphView g = v;
        g.q = qSoA;
        cellPrimitives<<<gridFor(v.all, 256), 256, 0, s>>>(g, 0, v.all);
        launched();
    }
    void launchWale(cudaStream_t s, const ReactiveTransportState* state) {
        GraphView g = v;
        g.state = state;
        cellGradients<<<gridFor(v.cells, 256), 256, 0, s>>>(g);
        launched();
        cellWale<<<gridFor(v.cells, 256), 256, 0, s>>>(g);
        launched();
        ++waleProfile.gradientBuilds;
        ++waleProfile.viscosityBuilds;
        waleProfile.cellsEvaluated += v.cells;
    }
    void buildWaleChecked() {
        if (!v.wale) return;
        check(cudaMemsetAsync(flags, 0, sizeof(unsigned), stream), "memset");
        if (structured) launchHostBoxGradients();
        else launchWale(stream, stateDevice);
        unsigned status = 0;
        download(&status, flags, 1);
        finish();
        require(!status, "Invalid WALE gradient/filter width/eddy viscosity");
    }
    // Face work (+ gradients) for one flux evaluation on device data.
    void launchFaces(const double* qSoA, const ReactiveTransportState* state, cudaStream_t s) {
        GraphView g = v;
        g.q = qSoA;
        g.state = state;
        if (v.wale) launchWale(s, state);
        else if (cfg.viscosity > 0) {
            cellGradients<<<gridFor(v.cells, 256), 256, 0, s>>>(g);
            launched();
        }
        faceWork<<<gridFor(v.faces, 128), 128, 0, s>>>(g);
        launched();
        ++deviceProfile.transportFaceLaunches;
    }
    void launchRates(const double* qSoA, const ReactiveTransportState* state, double* out, size_t stride,
                     int mode, double dt, cudaStream_t s) {
        GraphView g = v;
        g.q = qSoA;
        g.state = state;
        cellRates<8><<<gridFor(v.cells, 128), 128, 0, s>>>(g, out, stride, mode, dt);
        launched();
    }
    void launchLedger(const double* qSoA, const ReactiveTransportState* state, double* rate, cudaStream_t s) {
        GraphView g = v;
        g.q = qSoA;
        g.state = state;
        boundaryLedger<<<unsigned(cfg.variables), 256, 0, s>>>(g, rate);
        launched();
    }
    void launchSpeeds(const ReactiveTransportState* state, cudaStream_t s) {
        GraphView g = v;
        g.state = state;
        faceSpeeds<<<gridFor(v.faces, 256), 256, 0, s>>>(g);
        launched();
        ++deviceProfile.cflFaceLaunches;
    }
    void launchStep(double cfl, double maximumStep, double* result, cudaStream_t s) {
        cellSteps<<<gridFor(v.cells, 256), 256, 0, s>>>(v, cfl, maximumStep);
        launched();
        const unsigned blocks = unsigned(reduceBlocks);
        minimumReduce<<<blocks, 256, 0, s>>>(v.step, v.cells, reduceScratch);
        launched();
        minimumReduce<<<1, 1024, 0, s>>>(reduceScratch, blocks, result);
        launched();
    }

    // ------------------------------------------------ structured Cartesian box
    // The face list is a uniform nx x ny x nz box in the canonical ordering:
    // cells in natural order c = i + nx (j + ny k); internal faces sorted by
    // (owner, neighbour) with owner the lower cell, normal exactly +e_axis,
    // ownerWeight 0.5 and one area and distance per axis; then the boundary
    // faces in six contiguous side blocks (-x, +x, -y, +y, -z, +z), each in
    // lateral order (fast, slow) = (j, k), (i, k), (i, j), normal exactly
    // -+e_axis. Any other face list, species diffusion, the mechanical
    // variables, or more than four species use the face graph.
    bool detectBox(const ReactiveTransportFace* faces, size_t nInternal, const double* invDevice,
                   const ReactiveTransportPrimitive* primitive) {
        if (cfg.mechanical || cfg.diffusivity != 0 || cfg.variables != cfg.species + 4 || cfg.species < 1
            || cfg.species > size_t(kCartMaxNs) || nInternal < 3 || cfg.cells < 8)
            return false;
        if (faces[1].neighbour <= 0 || faces[2].neighbour <= 0 || size_t(faces[2].neighbour) >= cfg.cells)
            return false;
        const size_t nx = size_t(faces[1].neighbour), nxy = size_t(faces[2].neighbour);
        if (faces[0].owner != 0 || faces[0].neighbour != 1 || faces[1].owner != 0 || faces[2].owner != 0 || nx < 2
            || nxy < 2 * nx || nxy % nx || cfg.cells % nxy)
            return false;
        const size_t ny = nxy / nx, nz = cfg.cells / nxy;
        if (ny < 2 || nz < 2 || nx > INT32_MAX || ny > INT32_MAX || nz > INT32_MAX) return false;
        const size_t internal = (nx - 1) * ny * nz + nx * (ny - 1) * nz + nx * ny * (nz - 1);
        const size_t bnd = 2 * (ny * nz + nx * nz + nx * ny);
        if (internal != nInternal || internal + bnd != cfg.faces) return false;
        double area[3] = {faces[0].area, faces[1].area, faces[2].area};
        double dist[3] = {faces[0].distance, faces[1].distance, faces[2].distance};
        auto axisNormal = [](const ReactiveTransportFace& f, int axis, double sgn) {
            for (int d = 0; d < 3; ++d)
                if (f.normal[d] != (d == axis ? sgn : 0.0)) return false;
            return true;
        };
        size_t fi = 0;
        for (size_t c = 0; c < cfg.cells; ++c) {
            const size_t i = c % nx, j = (c / nx) % ny, k = c / nxy;
            const bool has[3] = {i + 1 < nx, j + 1 < ny, k + 1 < nz};
            const size_t step[3] = {1, nx, nxy};
            for (int a = 0; a < 3; ++a) {
                if (!has[a]) continue;
                const auto& f = faces[fi++];
                if (size_t(f.owner) != c || f.neighbour < 0 || size_t(f.neighbour) != c + step[a] || f.kind != 0
                    || !axisNormal(f, a, 1.0) || f.area != area[a] || f.distance != dist[a] || f.ownerWeight != .5)
                    return false;
            }
        }
        size_t base[6];
        for (int side = 0; side < 6; ++side) {
            const int a = side >> 1;
            const bool upper = side & 1;
            const size_t fast = a == 0 ? ny : nx, slow = a == 2 ? ny : nz;
            base[side] = fi;
            for (size_t t = 0; t < slow; ++t)
                for (size_t u = 0; u < fast; ++u) {
                    size_t i = 0, j = 0, k = 0;
                    if (a == 0) { i = upper ? nx - 1 : 0; j = u; k = t; }
                    else if (a == 1) { j = upper ? ny - 1 : 0; i = u; k = t; }
                    else { k = upper ? nz - 1 : 0; i = u; j = t; }
                    const auto& f = faces[fi++];
                    if (size_t(f.owner) != i + nx * (j + ny * k) || f.neighbour != -1 || f.kind < 1 || f.kind > 3
                        || !axisNormal(f, a, upper ? 1.0 : -1.0))
                        return false;
                }
        }
        box.nx = int(nx); box.ny = int(ny); box.nz = int(nz);
        box.cells = cfg.cells; box.fixed = cfg.fixed; box.all = cfg.cells + cfg.fixed;
        for (int a = 0; a < 3; ++a) { box.area[a] = area[a]; box.dist[a] = dist[a]; }
        box.invV = invDevice;
        box.face = v.face;
        for (int side = 0; side < 6; ++side) box.sideBase[side] = base[side];
        box.boundaryBase = nInternal;
        box.nBoundary = bnd;
        box.primitive = primitive;
        box.viscosity = cfg.viscosity; box.conductivity = cfg.conductivity; box.waveFactor = cfg.waveFactor;
        return true;
    }
    // Own cells [begin, end) (reactive_transport_owned_cells_v3): the stage
    // update, the CFL minimum and the boundary ledger cover them only.
    void setOwned(size_t begin, size_t end) {
        require(begin < end && end <= cfg.cells, "Owned cell range must be non-empty and within the cells");
        v.ownBegin = begin;
        v.ownEnd = end;
    }
    int fluxScheme = 0;  // structured path: 0 HLL, 1 HLLC
    CartView boxView() const {
        CartView b = box;
        b.ownBegin = v.ownBegin;
        b.ownEnd = v.ownEnd;
        b.wale = v.wale;
        b.cw = v.cw;
        b.scheme = fluxScheme;
        b.sgs = v.sgs;
        b.pr = v.pr;
        b.sc = v.sc;
        b.mixCp = v.mixCp;
        b.spH = v.spH;
        // the split stage's face fluxes live in the face graph's workspace, which
        // the structured path leaves unused (capillary handles keep it for theirs)
        const size_t need = splitScratchDoubles(int(cfg.variables), b.cells, true);
        b.faceFlux = v.work && !v.capillary && need <= product(v.faces, FW_FIELDS) ? v.work : nullptr;
        return b;
    }
    template <template <int> class K, class... Args> void bySpecies(Args&&... args) {
        switch (cfg.species) {
        case 1: K<1>::run(std::forward<Args>(args)...); break;
        case 2: K<2>::run(std::forward<Args>(args)...); break;
        case 3: K<3>::run(std::forward<Args>(args)...); break;
        default: K<4>::run(std::forward<Args>(args)...); break;
        }
        launched();
    }
    // Block sizes of the structured kernels (reactive_transport_autotune_v3
    // times the candidates on the handle's own problem and keeps the fastest;
    // the results do not depend on them).
    struct BoxLaunch {
        // rates 0 selects the shared-memory tiled stage kernel, 1 the split stage
        // (the default: the fastest on the 160^3 box on B200, FP64 and mixed; it
        // runs the per-cell kernel where the face workspace cannot hold its
        // scratch), 64/96/128 the per-cell kernel; the autotuner times them all
        unsigned rates = 1, gradients = 128, steps = 256;
    } launch;
    template <int NS> struct GradientsK {
        template <class R>
        static void run(const CartView& b, const ReactiveTransportState* st, R* grad, R* nut, unsigned* error,
                        unsigned block, cudaStream_t s) {
            cartGradients<NS, R><<<gridFor(b.cells, block), block, 0, s>>>(b, st, grad, nut, error);
        }
    };
    template <int NS> struct RatesK {
        // The split stage (cartFaceFluxes, cartRatesFromFaces, cartRatesBoxSides)
        // in arithmetic type R; with cfl > 0 also the CFL step of the same state
        // into *result (cartSteps' minimum, from the same face speeds).
        template <class R>
        static void split(const CartView& b, const double* q, const ReactiveTransportState* st, const R* grad,
                          const R* nut, double* out, size_t stride, int mode, double dt, unsigned* error, double cfl,
                          double maximumStep, double* result, cudaStream_t s) {
            const bool cflPass = cfl > 0;
            const unsigned grid = gridFor(b.cells, 128), cellGrid = gridFor(b.cells, 256);
            if (b.sgs) cartFaceFluxes<NS, R, true><<<grid, 128, 0, s>>>(b, q, st, grad, nut, error, cflPass);
            else cartFaceFluxes<NS, R><<<grid, 128, 0, s>>>(b, q, st, grad, nut, error, cflPass);
            cartRatesFromFaces<NS, R><<<cellGrid, 256, 0, s>>>(b, q, out, stride, mode, dt, cfl, maximumStep);
            const bool shell = b.nx >= 3 && b.ny >= 3 && b.nz >= 3;
            const size_t sides = shell ? 2 * size_t(b.nx) * b.ny
                                             + size_t(b.nz - 2) * (2 * size_t(b.nx) + 2 * size_t(b.ny - 2))
                                       : b.cells;
            const unsigned sideGrid = gridFor(sides, 128);
            if (b.sgs)
                cartRatesBoxSides<NS, R, true><<<sideGrid, 128, 0, s>>>(b, q, st, grad, nut, out, stride, mode, dt,
                                                                       error, cfl, maximumStep, cellGrid);
            else
                cartRatesBoxSides<NS, R><<<sideGrid, 128, 0, s>>>(b, q, st, grad, nut, out, stride, mode, dt, error,
                                                                 cfl, maximumStep, cellGrid);
            if (cflPass)
                minimumReduce<<<1, 1024, 0, s>>>(b.faceFlux + splitStepOffset(NQ, b.cells), size_t(cellGrid) + sideGrid,
                                                 result);
        }
        static constexpr int NQ = NS + 4;
        // block 0: the shared-memory tiled kernel; 1: the split stage;
        // otherwise the per-cell kernel with that many threads a block (all give
        // the same bits)
        template <class R, bool SGS>
        static void tiled(const CartView& b, const double* q, const ReactiveTransportState* st, const R* grad,
                          const R* nut, double* out, size_t stride, int mode, double dt, unsigned* error,
                          cudaStream_t s) {
            const size_t bytes = TileLayout<NS, SGS>::template bytes<R>();
            static thread_local int configured = -1;
            int device = 0;
            check(cudaGetDevice(&device), "cudaGetDevice");
            if (configured != device) {
                check(cudaFuncSetAttribute(cartRatesTile<NS, R, SGS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           int(bytes)),
                      "tiled stage shared memory");
                configured = device;
            }
            const dim3 grid((b.nx + kTileX - 1) / kTileX, (b.ny + kTileY - 1) / kTileY,
                            (b.nz + kTileZ - 1) / kTileZ);
            cartRatesTile<NS, R, SGS><<<grid, kTileX * kTileY, bytes, s>>>(b, q, st, grad, nut, out, stride, mode, dt,
                                                                         error);
        }
        template <class R>
        static void run(const CartView& b, const double* q, const ReactiveTransportState* st, const R* grad,
                        const R* nut, double* out, size_t stride, int mode, double dt, unsigned* error,
                        unsigned block, cudaStream_t s) {
            // block 1: the split stage (face fluxes once, then the per-cell sums; the
            // same bits); without its scratch, 128 threads per cell
            if (block == 1) {
                if (b.faceFlux) {
                    split<R>(b, q, st, grad, nut, out, stride, mode, dt, error, 0.0, 0.0, nullptr, s);
                    return;
                }
                block = 128;
            }
            if (block == 0) {
                if (b.sgs) tiled<R, true>(b, q, st, grad, nut, out, stride, mode, dt, error, s);
                else tiled<R, false>(b, q, st, grad, nut, out, stride, mode, dt, error, s);
                return;
            }
            if (b.sgs)
                cartRates<NS, R, true><<<gridFor(b.cells, block), block, 0, s>>>(b, q, st, grad, nut, out, stride,
                                                                               mode, dt, error);
            else
                cartRates<NS, R><<<gridFor(b.cells, block), block, 0, s>>>(b, q, st, grad, nut, out, stride, mode,
                                                                         dt, error);
        }
    };
    template <int NS> struct SplitK {
        template <class R>
        static void run(const CartView& b, const double* q, const ReactiveTransportState* st, const R* grad,
                        const R* nut, double* out, size_t stride, int mode, double dt, unsigned* error, double cfl,
                        double maximumStep, double* result, cudaStream_t s) {
            RatesK<NS>::template split<R>(b, q, st, grad, nut, out, stride, mode, dt, error, cfl, maximumStep, result,
                                          s);
        }
    };
    template <int NS> struct StepsK {
        template <class R>
        static void run(const CartView& b, const ReactiveTransportState* st, const R* nut, double cfl,
                        double maximumStep, double* partial, unsigned blocks, unsigned block, cudaStream_t s) {
            if (b.sgs) cartSteps<NS, R, true><<<blocks, block, 0, s>>>(b, st, nut, cfl, maximumStep, partial);
            else cartSteps<NS, R><<<blocks, block, 0, s>>>(b, st, nut, cfl, maximumStep, partial);
        }
    };
    template <int NS> struct LedgerK {
        template <class R>
        static void run(const CartView& b, const double* q, const ReactiveTransportState* st, const R* grad,
                        const R* nut, double* partial, unsigned blocks, cudaStream_t s) {
            if (b.sgs) cartLedger<NS, R, true><<<blocks, 256, 0, s>>>(b, q, st, grad, nut, partial);
            else cartLedger<NS, R><<<blocks, 256, 0, s>>>(b, q, st, grad, nut, partial);
        }
    };
    // Gradient (+ WALE viscosity) of the structured box, when the operator needs it.
    template <class R> void launchBoxGradientsT(const ReactiveTransportState* state, R* grad, R* nut, cudaStream_t s) {
        if (!(v.wale || cfg.viscosity > 0)) return;
        bySpecies<GradientsK>(boxView(), state, grad, nut, flags, launch.gradients, s);
        if (v.wale) {
            ++waleProfile.gradientBuilds;
            ++waleProfile.viscosityBuilds;
            waleProfile.cellsEvaluated += v.cells;
        }
    }
    // gradientsReady: the gradients and eddy viscosities of `state` (and the
    // primitives of qIn) were formed by the preceding launches on this stream.
    template <class R>
    void launchBoxStageT(const double* qIn, double* qOut, const ReactiveTransportState* state, double dt, int stage,
                         double* rate, R* grad, R* nut, cudaStream_t s, bool gradientsReady = false) {
        if (!gradientsReady) launchBoxGradientsT(state, grad, nut, s);
        if (rate) {
            bySpecies<LedgerK>(boxView(), qIn, state, static_cast<const R*>(grad), static_cast<const R*>(nut),
                               ledgerPartial, ledgerBlocks, s);
            foldPartials<<<1, 32 * unsigned(cfg.variables), 0, s>>>(ledgerPartial, int(ledgerBlocks),
                                                                    int(cfg.variables), rate);
            launched();
        }
        bySpecies<RatesK>(boxView(), qIn, state, static_cast<const R*>(grad), static_cast<const R*>(nut), qOut, v.all,
                          stage == 0 ? 1 : 2, dt, flags, launch.rates, s);
        ++deviceProfile.transportFaceLaunches;
    }
    template <class R>
    void launchBoxStepT(const ReactiveTransportState* state, double cfl, double maximumStep, double* result, R* grad,
                        R* nut, cudaStream_t s) {
        if (v.wale) launchBoxGradientsT(state, grad, nut, s);
        const unsigned blocks = unsigned(reduceBlocks);
        bySpecies<StepsK>(boxView(), state, static_cast<const R*>(nut), cfl, maximumStep, reduceScratch, blocks,
                          launch.steps, s);
        ++deviceProfile.cflFaceLaunches;
        minimumReduce<<<1, 1024, 0, s>>>(reduceScratch, blocks, result);
        launched();
    }
    void launchBoxStage(const double* qIn, double* qOut, const ReactiveTransportState* state, double dt, int stage,
                        double* rate, cudaStream_t s) {
        if (mixed) launchBoxStageT(qIn, qOut, state, dt, stage, rate, gradF, nutF, s);
        else launchBoxStageT(qIn, qOut, state, dt, stage, rate, v.grad, v.nut, s);
    }
    // The CFL query and then the stage on the same state: the CFL pass forms the
    // gradients and eddy viscosities when WALE is on, and the stage reuses them.
    void launchBoxStepStage(const double* qIn, double* qOut, const ReactiveTransportState* state, double dt,
                            int stage, double* rate, double cfl, double maximumStep, double* result, cudaStream_t s) {
        if (launch.rates == 1 && boxView().faceFlux) {
            // the split stage forms the CFL step of the same state with its fluxes
            if (mixed) launchSplitStepStage(qIn, qOut, state, dt, stage, rate, cfl, maximumStep, result, gradF, nutF, s);
            else launchSplitStepStage(qIn, qOut, state, dt, stage, rate, cfl, maximumStep, result, v.grad, v.nut, s);
            return;
        }
        launchBoxStep(state, cfl, maximumStep, result, s);
        if (mixed) launchBoxStageT(qIn, qOut, state, dt, stage, rate, gradF, nutF, s, v.wale);
        else launchBoxStageT(qIn, qOut, state, dt, stage, rate, v.grad, v.nut, s, v.wale);
    }
    template <class R>
    void launchSplitStepStage(const double* qIn, double* qOut, const ReactiveTransportState* state, double dt,
                              int stage, double* rate, double cfl, double maximumStep, double* result, R* grad,
                              R* nut, cudaStream_t s) {
        const CartView b = boxView();
        launchBoxGradientsT(state, grad, nut, s);
        if (rate) {
            bySpecies<LedgerK>(b, qIn, state, static_cast<const R*>(grad), static_cast<const R*>(nut), ledgerPartial,
                               ledgerBlocks, s);
            foldPartials<<<1, 32 * unsigned(cfg.variables), 0, s>>>(ledgerPartial, int(ledgerBlocks),
                                                                    int(cfg.variables), rate);
            launched();
        }
        bySpecies<SplitK>(b, qIn, state, static_cast<const R*>(grad), static_cast<const R*>(nut), qOut, v.all,
                          stage == 0 ? 1 : 2, dt, flags, cfl, maximumStep, result, s);
        ++deviceProfile.cflFaceLaunches;
        ++deviceProfile.transportFaceLaunches;
    }
    void launchBoxStep(const ReactiveTransportState* state, double cfl, double maximumStep, double* result,
                       cudaStream_t s) {
        if (mixed) launchBoxStepT(state, cfl, maximumStep, result, gradF, nutF, s);
        else launchBoxStepT(state, cfl, maximumStep, result, v.grad, v.nut, s);
    }
    template <int NS> struct RateVjpK {
        static void run(const CartView& b, const double* q, const ReactiveTransportState* st, const double* grad,
                        const double* nut, const double* w, double* qBar, ReactiveTransportState* stateBar,
                        double* gBar, double* nutBar, bool viscous, cudaStream_t s) {
            // the state-side derivatives: HLL by hand (with the viscous and conduction
            // terms at fixed gradients), HLLC in dual numbers
            if (b.scheme == 0)
                cartRateVjpInviscid<NS><<<gridFor(b.cells, 128), 128, 0, s>>>(b, q, st, grad, nut, w, qBar, stateBar);
            else
                cartRateVjp<NS, 0><<<gridFor(b.cells, 128), 128, 0, s>>>(b, q, st, grad, nut, w, qBar, stateBar,
                                                                        nullptr, nullptr);
            if (!viscous) return;
            cartViscousGradVjp<NS><<<gridFor(b.cells, 128), 128, 0, s>>>(b, q, st, grad, nut, w, gBar, nutBar);
            if (b.wale) cartWaleVjp<<<gridFor(b.cells, 128), 128, 0, s>>>(b, grad, nutBar, gBar);
            cartGradientVjp<NS><<<gridFor(b.cells, 256), 256, 0, s>>>(b, q, gBar, qBar);
        }
    };
    double* gradBar = nullptr;  // 9 x cells, rate VJP scratch
    double* nutBarBuf = nullptr;
    // (dL/dq)^T w and (dL/dstate)^T w of the FP64 structured operator at q: the
    // forward gradient and eddy viscosity are rebuilt from q first.
    void launchRateVjp(const double* q, const ReactiveTransportState* state, const double* w, double* qBar,
                       ReactiveTransportState* stateBar, cudaStream_t s) {
        require(structured, "The rate VJP needs the structured Cartesian path (reactive_transport_structured_v3)");
        require(!v.sgs, "The rate VJP does not cover the WALE scalar closure");
        const bool viscous = cfg.viscosity > 0 || v.wale;
        if (viscous && !gradBar) {
            gradBar = arena.get<double>(product(cfg.cells, 9));
            nutBarBuf = arena.get<double>(cfg.cells);
        }
        launchPrimitives(q, s);
        if (viscous) launchBoxGradientsT(state, v.grad, v.nut, s);
        bySpecies<RateVjpK>(boxView(), q, state, static_cast<const double*>(v.grad), static_cast<const double*>(v.nut),
                            w, qBar, stateBar, gradBar, nutBarBuf, viscous, s);
    }
    // Times each candidate block size on this handle's problem (q, state as
    // the device stage entries take them) and keeps the fastest; synchronous.
    void autotune(const double* q, const ReactiveTransportState* state, cudaStream_t s, unsigned* chosen) {
        require(structured, "Autotuning covers the structured path (reactive_transport_structured_v3)");
        double* out = arena.get<double>(product(v.all, cfg.variables));
        check(cudaMemcpyAsync(out, q, product(v.all, cfg.variables) * sizeof(double), cudaMemcpyDeviceToDevice, s),
              "copy");
        cudaEvent_t a, b;
        check(cudaEventCreate(&a), "event");
        check(cudaEventCreate(&b), "event");
        auto timeIt = [&](auto&& body) {
            body();  // warm-up
            float best = 1e30f;
            for (int r = 0; r < 3; ++r) {
                check(cudaEventRecord(a, s), "event");
                body();
                check(cudaEventRecord(b, s), "event");
                check(cudaEventSynchronize(b), "event");
                float ms = 0;
                check(cudaEventElapsedTime(&ms, a, b), "event");
                best = std::min(best, ms);
            }
            return best;
        };
        auto pick = [&](unsigned& slot, std::initializer_list<unsigned> candidates, auto&& body) {
            float best = 1e30f;
            unsigned keep = slot;
            for (unsigned c : candidates) {
                slot = c;
                const float t = timeIt(body);
                if (t < best) { best = t; keep = c; }
            }
            slot = keep;
        };
        launchPrimitives(q, s);
        // candidates stay within each kernel's __launch_bounds__ (128 for the stage, 256 otherwise)
        pick(launch.gradients, {64u, 128u, 256u}, [&] {
            if (mixed) launchBoxGradientsT(state, gradF, nutF, s);
            else launchBoxGradientsT(state, v.grad, v.nut, s);
        });
        pick(launch.rates, {0u, 1u, 64u, 96u, 128u}, [&] { launchBoxStage(q, out, state, 1e-30, 0, nullptr, s); });
        pick(launch.steps, {64u, 128u, 256u}, [&] { launchBoxStep(state, .5, 1.0, reduceScratch + reduceBlocks, s); });
        check(cudaEventDestroy(a), "event");
        check(cudaEventDestroy(b), "event");
        check(cudaStreamSynchronize(s), "sync");
        if (chosen) { chosen[0] = launch.rates; chosen[1] = launch.gradients; chosen[2] = launch.steps; }
    }
    // Mixed precision of the structured path: FP32 gradients, WALE and face
    // fluxes, compensated per-cell sums, FP64 conserved state and update.
    void setMixed(bool on) {
        if (on) {
            require(structured, "Mixed precision needs the structured Cartesian path (reactive_transport_structured_v3)");
            if (!gradF) gradF = arena.get<float>(product(cfg.cells, 9));
            if (!nutF) nutF = arena.get<float>(cfg.cells);
        }
        mixed = on;
    }

    // ------------------------------------------------------- reference contract
    void prepareResident(const ReactiveTransportState* states, const double* gasY, const double* gasH, bool transport) {
        requireCapillaryGeometry();
        requireScalarFields(transport);
        requireWalePrEpoch(transport);
        if (!structured) ensureGraphScalarWork();
        uploadState(states);
        if (transport && cfg.diffusivity > 0) {
            packInto(const_cast<double*>(v.gasY), gasY, cfg.cells, cfg.species, v.all, 0);
            packInto(const_cast<double*>(v.gasH), gasH, cfg.cells, cfg.species, v.all, 0);
            profile.gasUploadBytes += 2 * cfg.cells * cfg.species * sizeof(double);
        }
        launchPrimitives(q, stream);
        if (v.wale) buildWaleChecked();
        if (structured) {
            // the host-array entries on the structured box: FP64 HLL stencils, bitwise
            // equal to the face graph; rates, ledger and CFL are formed by the caller steps
            if (!v.wale && cfg.viscosity > 0) launchHostBoxGradients();
            return;
        }
        if (transport) {
            GraphView g = v;
            if (!v.wale && cfg.viscosity > 0) {
                cellGradients<<<gridFor(v.cells, 256), 256, 0, stream>>>(g);
                launched();
            }
            if (v.capillary) check(cudaMemsetAsync(flags, 0, sizeof(unsigned), stream), "memset");
            faceWork<<<gridFor(v.faces, 128), 128, 0, stream>>>(g);
            launched();
            ++deviceProfile.transportFaceLaunches;
            if (v.wale || v.capillary) {
                unsigned status = 0;
                download(&status, flags, 1);
                finish();
                if (v.capillary) {
                    require(!(status & kCapillaryBit), "Invalid capillary face flux");
                    capillaryProfile.faceFluxBuilds += cfg.faces;
                }
                require(!(status & ~kCapillaryBit), "Nonfinite WALE traction/energy flux; stage remains uncommitted");
            }
        } else launchSpeeds(stateDevice, stream);
    }
    void prepare(const double* hostQ, const ReactiveTransportState* states, const double* gasY, const double* gasH,
                 bool transport) {
        haveResident = false;
        uploadQ(hostQ);
        prepareResident(states, gasY, gasH, transport);
    }
    void gather(bool materialize) {
        if (materialize && !rhs) rhs = arena.get<double>(product(cfg.cells, cfg.variables));
        if (structured) {
            const CartView b = hostBoxView();
            if (materialize) {
                if (v.wale) check(cudaMemsetAsync(flags, 0, sizeof(unsigned), stream), "memset");
                bySpecies<RatesK>(b, static_cast<const double*>(q), static_cast<const ReactiveTransportState*>(
                                      stateDevice), static_cast<const double*>(v.grad),
                                  static_cast<const double*>(v.nut), rhs, size_t(cfg.cells), 0, 0.0, flags,
                                  launch.rates, stream);
                ++deviceProfile.transportFaceLaunches;
                requireFiniteTraction();
            }
            bySpecies<LedgerK>(b, static_cast<const double*>(q), static_cast<const ReactiveTransportState*>(
                                   stateDevice), static_cast<const double*>(v.grad), static_cast<const double*>(v.nut),
                               ledgerPartial, ledgerBlocks, stream);
            foldPartials<<<1, 32 * unsigned(cfg.variables), 0, stream>>>(ledgerPartial, int(ledgerBlocks),
                                                                          int(cfg.variables), boundaryRate);
            launched();
            return;
        }
        if (materialize) launchRates(q, stateDevice, rhs, cfg.cells, 0, 0, stream);
        launchLedger(q, stateDevice, boundaryRate, stream);
    }
    // The structured view the host-array entries use: FP64 HLL whatever the
    // device entries' precision and flux scheme.
    CartView hostBoxView() const {
        CartView b = boxView();
        b.scheme = 0;
        return b;
    }
    void launchHostBoxGradients() {
        bySpecies<GradientsK>(hostBoxView(), static_cast<const ReactiveTransportState*>(stateDevice), v.grad, v.nut,
                              flags, launch.gradients, stream);
        if (v.wale) {
            ++waleProfile.gradientBuilds;
            ++waleProfile.viscosityBuilds;
            waleProfile.cellsEvaluated += v.cells;
        }
    }
    // A non-finite WALE traction or energy flux fails the call before anything
    // is committed (the face graph checks the same after its face pass).
    void requireFiniteTraction() {
        if (!v.wale) return;
        unsigned status = 0;
        download(&status, flags, 1);
        finish();
        require(!(status & 1u), "Nonfinite WALE traction/energy flux; stage remains uncommitted");
    }
    void stableStep(double cfl, double maximumStep, double* dt) {
        require(dt && std::isfinite(cfl) && cfl > 0 && cfl <= .5 && std::isfinite(maximumStep) && maximumStep > 0,
                "Invalid transport CFL controls");
        if (structured) {
            const unsigned blocks = unsigned(reduceBlocks);
            bySpecies<StepsK>(hostBoxView(), static_cast<const ReactiveTransportState*>(stateDevice),
                              static_cast<const double*>(v.nut), cfl, maximumStep, reduceScratch, blocks, launch.steps,
                              stream);
            ++deviceProfile.cflFaceLaunches;
            minimumReduce<<<1, 1024, 0, stream>>>(reduceScratch, blocks, reduceScratch + reduceBlocks);
            launched();
        } else launchStep(cfl, maximumStep, reduceScratch + reduceBlocks, stream);
        download(dt, reduceScratch + reduceBlocks, 1);
        finish();
        require(std::isfinite(*dt) && *dt > 0, "Invalid wave/diffusion timestep");
        ++stats.stepQueries;
    }
    void advance(double dt, int stage, double* hostQ, double* boundary) {
        if (structured) {
            if (v.wale) check(cudaMemsetAsync(flags, 0, sizeof(unsigned), stream), "memset");
            bySpecies<RatesK>(hostBoxView(), static_cast<const double*>(q),
                              static_cast<const ReactiveTransportState*>(stateDevice),
                              static_cast<const double*>(v.grad), static_cast<const double*>(v.nut), initial, v.all,
                              stage == 0 ? 1 : 2, dt, flags, launch.rates, stream);
            ++deviceProfile.transportFaceLaunches;
            requireFiniteTraction();
        } else launchRates(q, stateDevice, initial, v.all, stage == 0 ? 1 : 2, dt, stream);
        std::swap(q, initial);
        v.q = q;
        if (hostQ) unpackQ(hostQ);
        download(boundary, boundaryRate, cfg.variables);
        finish();
        haveInitial = stage == 0;
        stageDt = dt;
        ++stats.stages;
    }
    // Diffuse capillary closure (src/reactiveTransport/reactiveTransport.cpp:859-886).
    void setCapillary(const ReactiveCapillaryOptionsV1& options) {
        require(options.abiVersion == 1 && options.structBytes == sizeof(options) && std::isfinite(options.sigma)
                    && options.sigma > 0 && std::isfinite(options.capillaryCfl) && options.capillaryCfl > 0
                    && options.capillaryCfl <= 1 && std::isfinite(options.geometryEpsilon)
                    && options.geometryEpsilon >= 0 && options.geometryEpsilon < 1,
                "Invalid capillary options ABI/model");
        require(!v.capillary && !attemptOpen && !stats.stages && !highestVersion,
                "Capillary model must be installed once before stepping");
        require(!cfg.mechanical && cfg.variables == cfg.species + 5 && options.condensableSpecies >= 0
                    && size_t(options.condensableSpecies) < cfg.species,
                "Capillary model needs one mapped conserved liquid inventory");
        const size_t before = arena.bytes;
        // one block: color (all), gradient and normal (3 x cells each), area
        // density, curvature and surface energy (cells each)
        double* block = arena.get<double>(v.all + product(cfg.cells, 9));
        check(cudaMemsetAsync(block, 0, (v.all + product(cfg.cells, 9)) * sizeof(double), stream), "memset");
        colorDevice = block;
        v.color = block;
        v.cGrad = block + v.all;
        v.cNormal = v.cGrad + 3 * cfg.cells;
        v.cArea = v.cNormal + 3 * cfg.cells;
        v.cCurv = v.cArea + cfg.cells;
        v.cEnergy = v.cCurv + cfg.cells;
        v.capError = flags;
        v.sigma = options.sigma;
        v.capCfl = options.capillaryCfl;
        v.geomEps = options.geometryEpsilon;
        v.capSpecies = size_t(options.condensableSpecies);
        v.capillary = true;
        finish();
        capillaryProfile.capillaryWorkspaceBytes = arena.bytes - before + sizeof(uint32_t);
    }
    // src/reactiveTransport/reactiveTransport.cpp:887-962 (diffuse geometry).
    void capillaryGeometry(const double* cellColor, const double* fixedColor, double* energy, double* curvature,
                           double* normal) {
        require(v.capillary && cellColor && energy && (!cfg.fixed || fixedColor),
                "Missing capillary model, color or surface-energy output");
        const auto unit = [](double c) { return std::isfinite(c) && c >= 0 && c <= 1; };
        require(firstFailure(cfg.cells, [&](size_t c) { return unit(cellColor[c]); }) == cfg.cells,
                "Invalid material color");
        for (size_t c = 0; c < cfg.fixed; ++c) require(unit(fixedColor[c]), "Invalid fixed material color");
        retireWalePr();
        const auto same = [](const std::vector<double>& shadow, const double* x, size_t n) {
            return shadow.size() == n && (n == 0 || std::memcmp(shadow.data(), x, n * sizeof(double)) == 0);
        };
        if (!normal && colorReady && geometryShadowValid && (!curvature || !curvatureShadow.empty())
            && same(colorShadow, cellColor, cfg.cells) && same(fixedColorShadow, fixedColor, cfg.fixed)) {
            std::memcpy(energy, energyShadow.data(), cfg.cells * sizeof(double));
            if (curvature) std::memcpy(curvature, curvatureShadow.data(), cfg.cells * sizeof(double));
            ++geometryBuildsSkipped;
            return;
        }
        geometryShadowValid = false;
        colorReady = false;
        check(cudaMemsetAsync(flags, 0, sizeof(unsigned), stream), "memset");
        upload(colorDevice, cellColor, cfg.cells);
        upload(colorDevice + cfg.cells, fixedColor, cfg.fixed);
        const uint64_t previousKernels = stats.kernelLaunches;
        const unsigned blocks = unsigned(std::min<size_t>((cfg.cells + 255) / 256, 148 * 16));
        interfaceGradient<<<blocks, 256, 0, stream>>>(v);
        launched();
        interfaceCurvature<<<blocks, 256, 0, stream>>>(v);
        launched();
        download(energy, v.cEnergy, cfg.cells);
        if (curvature) download(curvature, v.cCurv, cfg.cells);
        if (normal) download(normal, v.cNormal, product(cfg.cells, 3));
        unsigned status = 0;
        download(&status, flags, 1);
        finish();
        require(!(status & kCapillaryBit), "Invalid capillary geometry");
        colorReady = true;
        ++capillaryProfile.geometryBuilds;
        colorShadow.assign(cellColor, cellColor + cfg.cells);
        fixedColorShadow.assign(fixedColor, fixedColor + cfg.fixed);
        energyShadow.assign(energy, energy + cfg.cells);
        if (curvature) curvatureShadow.assign(curvature, curvature + cfg.cells);
        else curvatureShadow.clear();
        geometryShadowValid = true;
        capillaryProfile.geometryCells += cfg.cells;
        capillaryProfile.geometryKernels += stats.kernelLaunches - previousKernels;
        capillaryProfile.colorUploadBytes += (cfg.cells + cfg.fixed) * sizeof(double);
        capillaryProfile.geometryDownloadBytes +=
            cfg.cells * sizeof(double) * (1 + (curvature ? 1 : 0) + (normal ? 3 : 0));
    }
    // --------------------------------------------------- WALE PR properties
    void installWalePr(const ReactiveWalePrModelV1& o) {
        require(o.abiVersion == 1 && o.structBytes == sizeof(o) && o.modelImage
                    && o.modelBytes == sizeof(ReactiveB200HemModel),
                "Invalid WALE PR model ABI or image size");
        require(o.physicalModelHash[64] == 0 && std::strlen(o.physicalModelHash) == 64
                    && physicalHash == o.physicalModelHash,
                "WALE PR model identity differs from transport physical model");
        require(v.capillary && v.sgs && !walePrInstalled && !highestVersion && !stats.stages && !stats.stepQueries,
                "WALE PR device model must be installed on CUDA before stepping");
        ReactiveB200HemModel host;
        std::memcpy(&host, o.modelImage, sizeof(host));
        require(host.ns >= 1 && host.ns <= mix::kMaxNs && host.nl == 1 && host.condensedKind[0] == 0
                    && size_t(host.ns) == cfg.species && v.capSpecies == size_t(host.condensable[0])
                    && cfg.variables == cfg.species + 5 && host.phase[0].ns == host.ns && host.phase[1].ns == 1
                    && std::isfinite(host.vtol) && host.vtol > 0,
                "WALE PR model does not match the single-liquid capillary transport layout");
        if (v.pr > 0) {
            require(!cfg.fixed || o.fixedCp, "Missing fixed WALE heat capacities");
            for (size_t c = 0; c < cfg.fixed; ++c)
                require(std::isfinite(o.fixedCp[c]) && o.fixedCp[c] > 0, "Invalid fixed WALE heat capacity");
        }
        if (v.sc > 0) {
            require(!cfg.fixed || o.fixedSpeciesH, "Missing fixed WALE species enthalpies");
            for (size_t i = 0; i < cfg.fixed * cfg.species; ++i)
                require(std::isfinite(o.fixedSpeciesH[i]), "Invalid fixed WALE species enthalpy");
        }
        const size_t n = cfg.cells, ns = cfg.species;
        size_t bytes = sizeof(host) + sizeof(unsigned long long) + product(n, sizeof(ReactiveThermoState) + sizeof(double));
        if (v.sc > 0) bytes += 2 * product(product(n, ns), sizeof(double));
        require(double(arena.bytes) + double(bytes) <= arena.limit,
                "WALE PR property scratch exceeds transport memory budget");
        walePrModel = arena.get<ReactiveB200HemModel>(1);
        walePrStates = arena.get<ReactiveThermoState>(n);
        if (v.sc > 0) {
            walePrQ = arena.get<double>(product(n, ns));
            walePrH = arena.get<double>(product(n, ns));
            walePrHostQ.resize(product(n, ns));
        }
        walePrCp = arena.get<double>(n);
        walePrFailure = arena.get<unsigned long long>(1);
        upload(walePrModel, &host, 1);
        if (v.pr > 0) upload(const_cast<double*>(v.mixCp) + n, o.fixedCp, cfg.fixed);
        if (v.sc > 0) packInto(const_cast<double*>(v.spH), o.fixedSpeciesH, cfg.fixed, ns, v.all, n);
        finish();
        // a prior host scalar upload is never a valid device PR property epoch
        scalarCp = scalarH = false;
        walePrReady = false;
        walePrInstalled = true;
        walePrProfile.scratchBytes = bytes;
        walePrProfile.inputUploadBytes = sizeof(host) + cfg.fixed * (v.pr > 0 ? sizeof(double) : 0)
                                       + cfg.fixed * ns * (v.sc > 0 ? sizeof(double) : 0);
    }
    void prepareWalePr(const ReactiveWalePrEpochV1& epoch, const double* hq, size_t stride,
                       const ReactiveThermoState* states, bool statesUnchanged) {
        const auto begin = std::chrono::steady_clock::now();
        const bool reuse = statesUnchanged && walePrStatesCurrent;
        // no failed request may publish old properties or promise a reusable upload
        walePrStatesCurrent = false;
        walePrReady = false;
        scalarCp = scalarH = false;
        require(epoch.abiVersion == 1 && epoch.structBytes == sizeof(epoch)
                    && (epoch.enthalpies == 0 || epoch.enthalpies == 1) && epoch.thermoVersion > 0
                    && epoch.thermoVersion >= walePrLastThermoVersion && epoch.boundaryVersion == 1,
                "Invalid WALE PR property epoch");
        require(walePrInstalled && colorReady && states && epoch.geometryVersion == capillaryProfile.geometryBuilds,
                "WALE PR properties require installed model and current capillary geometry");
        constexpr uint64_t kCflStage = std::numeric_limits<uint64_t>::max();
        if (attemptOpen) {
            if (epoch.nextConserved.stageId == kCflStage)
                require(!epoch.enthalpies && epoch.nextConserved.attemptId == attemptId
                            && !epoch.nextConserved.contentVersion,
                        "Invalid WALE PR in-attempt CFL token");
            else
                require(epoch.nextConserved.attemptId == attemptId && epoch.nextConserved.stageId == tokenStage
                            && epoch.nextConserved.contentVersion > highestVersion,
                        "Stale WALE PR next-conserved token");
        } else
            require(!epoch.nextConserved.attemptId && !epoch.nextConserved.stageId
                        && !epoch.nextConserved.contentVersion,
                    "WALE PR CFL properties cannot claim an RK token");
        if (epoch.enthalpies) {
            require(v.sc > 0 && v.spH && walePrQ && walePrH, "WALE PR enthalpies require species mixing scratch");
            require(hq && stride == cfg.variables, "WALE PR enthalpies need full conserved rows");
            require(attemptOpen, "WALE PR enthalpies require an open RK attempt");
        }
        const size_t n = cfg.cells, ns = cfg.species;
        if (epoch.enthalpies)
            for (size_t c = 0; c < n; ++c)
                for (size_t k = 0; k < ns; ++k) walePrHostQ[c * ns + k] = hq[c * stride + k];
        const unsigned long long none = std::numeric_limits<unsigned long long>::max();
        unsigned long long failure = none;
        upload(walePrFailure, &none, 1);
        if (!reuse) upload(walePrStates, states, n);
        if (epoch.enthalpies) upload(walePrQ, walePrHostQ.data(), product(n, ns));
        walePrProfile.inputUploadBytes += sizeof(none) + (reuse ? 0 : n * sizeof(ReactiveThermoState))
                                        + (epoch.enthalpies ? product(n, ns) * sizeof(double) : 0);
        const unsigned blocks = unsigned(std::min<size_t>((n + 127) / 128, 148 * 32));
        walePrProperties<<<blocks, 128, 0, stream>>>(walePrModel, walePrQ, walePrStates, v.color, v.cCurv, v.sigma,
                                                     n, ns, walePrH, walePrCp, walePrFailure, epoch.enthalpies != 0);
        launched();
        ++walePrProfile.kernels;
        download(&failure, walePrFailure, 1);
        finish();
        walePrProfile.cells += n;
        if (failure != none) {
            ++walePrProfile.failures;
            throw std::runtime_error("WALE PR GPU property cell " + std::to_string(failure >> 8) + " status "
                                     + std::to_string(failure & 255));
        }
        walePrCommit<<<blocks, 128, 0, stream>>>(n, ns, v.all, walePrH, walePrCp, const_cast<double*>(v.spH),
                                                 const_cast<double*>(v.mixCp), epoch.enthalpies != 0, v.pr > 0);
        launched();
        ++walePrProfile.kernels;
        finish();
        scalarCp = true;
        scalarH = epoch.enthalpies != 0 || v.sc == 0;
        walePrReady = true;
        walePrEpoch = epoch;
        walePrStatesCurrent = true;
        walePrLastThermoVersion = epoch.thermoVersion;
        ++walePrProfile.builds;
        walePrProfile.wallSeconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - begin).count();
    }
    // The published PR properties belong to the stage (transport) or the CFL
    // query they were built for (src/reactiveTransport/reactiveTransport.cpp:1398-1430).
    void requireWalePrEpoch(bool transport) const {
        if (!walePrInstalled) return;
        constexpr uint64_t kCflStage = std::numeric_limits<uint64_t>::max();
        const ReactiveTransportToken& next = walePrEpoch.nextConserved;
        if (transport)
            require(walePrReady && next.attemptId == attemptId && next.stageId == tokenStage
                        && next.contentVersion == residentVersion
                        && walePrEpoch.geometryVersion == capillaryProfile.geometryBuilds
                        && (v.sc == 0 || walePrEpoch.enthalpies == 1),
                    "WALE PR properties have a stale conserved or geometry epoch");
        else
            require(walePrReady && walePrEpoch.geometryVersion == capillaryProfile.geometryBuilds
                        && walePrEpoch.enthalpies == 0
                        && (attemptOpen ? next.attemptId == attemptId && next.stageId == kCflStage
                                              && !next.contentVersion
                                        : !next.attemptId && !next.stageId && !next.contentVersion),
                    "WALE PR CFL heat capacity has a stale geometry or attempt epoch");
    }
    // A new geometry retires the properties built on the old one.
    void retireWalePr() {
        if (!walePrInstalled) return;
        walePrReady = false;
        scalarCp = scalarH = false;
    }
    // ------------------------------------------- resident capillary closure
    // (src/reactiveTransport/reactiveTransport.cpp:963-1127)
    unsigned residentGrid(size_t n) const { return unsigned(std::min<size_t>(65535, (n + 255) / 256)); }
    // All buffers or none: a budget or allocation failure frees what this call
    // allocated, so a retry starts from the same state.
    void residentAllocate(size_t species) {
        const size_t n = cfg.cells;
        if (resident.cells == n && resident.species == species) return;
        require(!resident.cells, "Resident capillary species count changed");
        require(species == cfg.species && n <= size_t(std::numeric_limits<int>::max()),
                "Resident capillary species/count exceeds the transport or sort layout");
        CapillaryResident r;
        std::vector<void*> fresh;
        uint64_t freshBytes = 0;
        auto get = [&](size_t bytes) -> void* {
            require(double(arena.bytes) + double(freshBytes) + double(bytes) <= arena.limit,
                    "Resident capillary closure exceeds the transport workspace budget");
            void* p = nullptr;
            check(cudaMalloc(&p, std::max<size_t>(bytes, 1)), "cudaMalloc");
            fresh.push_back(p);
            freshBytes += bytes;
            return p;
        };
        try {
            r.cells = n;
            r.species = species;
            r.q = static_cast<double*>(get(product(product(n, species), sizeof(double))));
            double** arrays[] = {&r.bulk, &r.energy, &r.color, &r.jump, &r.colorBefore, &r.jumpBefore,
                                 &r.energyBefore, &r.flashedColor, &r.flashedJump, &r.flashedEnergy};
            for (double** a : arrays) *a = static_cast<double*>(get(product(n, sizeof(double))));
            r.seed = static_cast<ReactiveThermoState*>(get(product(n, sizeof(ReactiveThermoState))));
            r.output = static_cast<ReactiveGpuHemOutputV1*>(get(product(n, sizeof(ReactiveGpuHemOutputV1))));
            r.capillary = static_cast<ReactiveGpuHemCapillaryInputV2*>(
                get(product(n, sizeof(ReactiveGpuHemCapillaryInputV2))));
            r.keys = static_cast<uint16_t*>(get(product(n, sizeof(uint16_t))));
            r.sortedKeys = static_cast<uint16_t*>(get(product(n, sizeof(uint16_t))));
            r.cells32 = static_cast<uint32_t*>(get(product(n, sizeof(uint32_t))));
            r.order = static_cast<uint32_t*>(get(product(n, sizeof(uint32_t))));
            r.scalars = static_cast<unsigned long long*>(get(2 * sizeof(unsigned long long)));
            r.flags = static_cast<unsigned*>(get(sizeof(unsigned)));
            check(cub::DeviceRadixSort::SortPairs(nullptr, r.sortBytes, r.keys, r.sortedKeys, r.cells32, r.order,
                                                  int(n), 0, 9, stream),
                  "sort size");
            r.sortTemp = get(std::max<size_t>(r.sortBytes, 1));
            capres::identity<<<residentGrid(n), 256, 0, stream>>>(n, r.cells32);
            launched();
            check(cudaMemsetAsync(r.output, 0, product(n, sizeof(ReactiveGpuHemOutputV1)), stream), "memset");
            finish();
        } catch (...) {
            cudaStreamSynchronize(stream);
            for (void* p : fresh) cudaFree(p);
            throw;
        }
        arena.blocks.insert(arena.blocks.end(), fresh.begin(), fresh.end());
        arena.bytes += freshBytes;
        arena.peak = std::max(arena.peak, arena.bytes);
        capillaryProfile.capillaryWorkspaceBytes += freshBytes;
        resident = std::move(r);
    }
    void residentClearFlags() {
        check(cudaMemsetAsync(resident.flags, 0, sizeof(unsigned), stream), "memset");
        check(cudaMemsetAsync(resident.scalars, 0, 2 * sizeof(unsigned long long), stream), "memset");
    }
    unsigned residentFlags(unsigned long long* scalars = nullptr) {
        unsigned f = 0;
        download(&f, resident.flags, 1);
        if (scalars) download(scalars, resident.scalars, 2);
        finish();
        return f;
    }
    // The diffuse geometry of the device color and the jump sigma*kappa.
    void residentGeometry() {
        auto& r = resident;
        const size_t n = cfg.cells;
        retireWalePr();
        geometryShadowValid = false;
        colorReady = false;
        check(cudaMemsetAsync(flags, 0, sizeof(unsigned), stream), "memset");
        check(cudaMemcpyAsync(colorDevice, r.color, n * sizeof(double), cudaMemcpyDeviceToDevice, stream), "D2D");
        ++deviceCopies;
        upload(colorDevice + n, r.fixedColor.data(), cfg.fixed);
        const unsigned blocks = unsigned(std::min<size_t>((n + 255) / 256, 148 * 16));
        interfaceGradient<<<blocks, 256, 0, stream>>>(v);
        launched();
        interfaceCurvature<<<blocks, 256, 0, stream>>>(v);
        launched();
        capres::pressureJump<<<residentGrid(n), 256, 0, stream>>>(n, r.sigma, v.cCurv, r.jump);
        check(cudaGetLastError(), "kernel launch");
        unsigned status = 0;
        download(&status, flags, 1);
        finish();
        require(!(status & kCapillaryBit), "Invalid capillary geometry");
        colorReady = true;
        ++capillaryProfile.geometryBuilds;
        capillaryProfile.geometryCells += n;
        capillaryProfile.geometryKernels += 2;
        capillaryProfile.colorUploadBytes += cfg.fixed * sizeof(double);
    }
    void residentBegin(size_t species, const double* hq, const double* liquid, const double* bulk,
                       const ReactiveThermoState* states, const double* fixedColor, double sigma, int equilibrium,
                       int* fallback) {
        require(v.capillary, "Resident capillary closure needs CUDA diffuse geometry");
        require(species > 0 && hq && liquid && bulk && states && fallback && (!cfg.fixed || fixedColor)
                    && std::isfinite(sigma) && (equilibrium == 0 || equilibrium == 1),
                "Invalid resident capillary input");
        for (size_t c = 0; c < cfg.fixed; ++c)
            require(std::isfinite(fixedColor[c]) && fixedColor[c] >= 0 && fixedColor[c] <= 1,
                    "Invalid fixed material color");
        residentAllocate(species);
        auto& r = resident;
        const size_t n = cfg.cells;
        r.sigma = sigma;
        r.equilibrium = equilibrium;
        r.ready = false;
        r.fixedColor.assign(fixedColor, fixedColor + cfg.fixed);
        residentClearFlags();
        upload(r.q, hq, product(n, species));
        upload(r.bulk, bulk, n);
        upload(r.seed, states, n);
        upload(r.energy, liquid, n);  // the liquid inventory, folded into the seeds below
        capres::seedStates<<<residentGrid(n), 256, 0, stream>>>(n, r.seed, r.energy, r.color, r.flags);
        check(cudaGetLastError(), "kernel launch");
        if ((*fallback = residentFlags() != 0)) return;
        residentGeometry();
        r.ready = true;
    }
    void residentSelect(int iteration, ReactiveCapillaryResidentViewV1& view, int* fallback) {
        auto& r = resident;
        const size_t n = cfg.cells;
        require(r.ready && fallback && view.abiVersion == 1 && view.structBytes == sizeof(view),
                "Resident capillary select out of order");
        residentClearFlags();
        capres::selectDirty<<<unsigned((n + 255) / 256), 256, 0, stream>>>(
            n, iteration == 0, r.equilibrium, int(r.species), r.q, r.seed, r.bulk, r.color, r.jump, v.cEnergy,
            r.colorBefore, r.jumpBefore, r.energyBefore, r.flashedColor, r.flashedJump, r.flashedEnergy, r.energy,
            r.capillary, r.keys, r.scalars, r.flags);
        check(cudaGetLastError(), "kernel launch");
        size_t bytes = r.sortBytes;
        check(cub::DeviceRadixSort::SortPairs(r.sortTemp, bytes, r.keys, r.sortedKeys, r.cells32, r.order, int(n), 0,
                                              9, stream),
              "sort");
        unsigned long long scalars[2] = {0, 0};
        if ((*fallback = residentFlags(scalars) != 0)) {
            r.ready = false;
            return;
        }
        view.q = r.q;
        view.energy = r.energy;
        view.seed = r.seed;
        view.capillary = r.capillary;
        view.order = r.order;
        view.output = r.output;
        view.count = size_t(scalars[0]);
    }
    void residentUpdate(size_t count, double* residual, int* fallback) {
        auto& r = resident;
        const size_t n = cfg.cells;
        require(r.ready && residual && fallback && count <= n, "Resident capillary update out of order");
        residentClearFlags();
        if (count) {
            capres::recordFlashed<<<residentGrid(count), 256, 0, stream>>>(count, r.order, r.colorBefore,
                                                                          r.jumpBefore, r.energyBefore, r.flashedColor,
                                                                          r.flashedJump, r.flashedEnergy);
            check(cudaGetLastError(), "kernel launch");
        }
        capres::candidateColor<<<residentGrid(n), 256, 0, stream>>>(n, r.output, r.color, r.flags);
        check(cudaGetLastError(), "kernel launch");
        if ((*fallback = residentFlags() != 0)) {
            r.ready = false;
            return;
        }
        residentGeometry();
        capres::closureResidual<<<unsigned((n + 255) / 256), 256, 0, stream>>>(
            n, r.color, r.colorBefore, v.cEnergy, r.energyBefore, r.jump, r.jumpBefore, r.bulk, r.output,
            r.scalars + 1, r.flags);
        check(cudaGetLastError(), "kernel launch");
        unsigned long long scalars[2] = {0, 0};
        if ((*fallback = residentFlags(scalars) != 0)) {
            r.ready = false;
            return;
        }
        std::memcpy(residual, &scalars[1], sizeof(double));
    }
    void residentRelax() {
        auto& r = resident;
        require(r.ready, "Resident capillary relaxation out of order");
        capres::relaxColor<<<residentGrid(cfg.cells), 256, 0, stream>>>(cfg.cells, r.colorBefore, r.color);
        check(cudaGetLastError(), "kernel launch");
        residentGeometry();
    }
    void residentCommit(ReactiveThermoState* states, double* color, double* energy, double* curvature) {
        auto& r = resident;
        const size_t n = cfg.cells;
        require(r.ready && states && color && energy && curvature, "Resident capillary commit out of order");
        // the closure is over: the seed buffer stages the states' download
        capres::gatherStates<<<residentGrid(n), 256, 0, stream>>>(n, r.output, r.seed);
        check(cudaGetLastError(), "kernel launch");
        download(states, r.seed, n);
        download(color, r.color, n);
        download(energy, v.cEnergy, n);
        download(curvature, v.cCurv, n);
        finish();
        capillaryProfile.geometryDownloadBytes += n * 2 * sizeof(double);
        // the published geometry is exactly the build of `color`: a later
        // identical host request reuses it
        colorShadow.assign(color, color + n);
        fixedColorShadow = r.fixedColor;
        energyShadow.assign(energy, energy + n);
        curvatureShadow.assign(curvature, curvature + n);
        geometryShadowValid = true;
        r.ready = false;
    }
    void installWale(const ReactiveWaleOptionsV1& options) {
        require(options.abiVersion == 1 && options.structBytes == sizeof(options), "Invalid WALE options ABI");
        require(!v.wale && !highestVersion && !stats.stages && !stats.stepQueries && profile.conservedUploads == 0
                    && profile.stateUploadBytes == 0,
                "WALE is immutable and must be installed before stepping");
        require(!cfg.mechanical, "WALE mechanical-environment closure is not implemented");
        require(std::isfinite(options.Cw) && options.Cw >= 0, "Invalid WALE coefficient");
        const size_t before = arena.bytes;
        if (!v.grad) v.grad = arena.get<double>(product(cfg.cells, 9));
        v.nut = arena.get<double>(cfg.cells);
        v.cw = options.Cw;
        v.wale = true;
        waleProfile.workspaceBytes = arena.bytes - before + sizeof(uint32_t);
    }
    // WALE scalar closure (src/reactiveTransport/reactiveTransport.cpp:653-702).
    void installWaleScalars(const ReactiveWaleScalarOptionsV1& options) {
        require(options.abiVersion == 1 && options.structBytes == sizeof(options), "Invalid WALE scalar options ABI");
        require(v.wale && !v.sgs && !highestVersion && !stats.stages && !stats.stepQueries
                    && profile.conservedUploads == 0 && profile.stateUploadBytes == 0,
                "WALE scalar closure is immutable and must be installed before stepping");
        require(!cfg.mechanical, "WALE scalar mechanical-environment closure is not implemented");
        require(std::isfinite(options.turbulentPrandtl) && std::isfinite(options.turbulentSchmidt)
                    && options.turbulentPrandtl >= 0 && options.turbulentSchmidt >= 0,
                "Invalid turbulent Prandtl/Schmidt number");
        require(options.turbulentSchmidt == 0 || cfg.variables == cfg.species + 4
                    || (v.capillary && cfg.variables == cfg.species + 5 && v.capSpecies < cfg.species),
                "WALE total-species mixing requires equilibrium phase partition or a mapped capillary liquid "
                "inventory; frozen non-capillary inventories are unsupported");
        const size_t before = arena.bytes;
        if (options.turbulentPrandtl > 0) v.mixCp = arena.get<double>(v.all);
        if (options.turbulentSchmidt > 0) {
            double* h = arena.get<double>(product(v.all, cfg.species));
            check(cudaMemsetAsync(h, 0, product(v.all, cfg.species) * sizeof(double), stream), "memset");
            v.spH = h;
        }
        v.pr = options.turbulentPrandtl;
        v.sc = options.turbulentSchmidt;
        v.sgs = true;
        if (!structured) ensureGraphScalarWork();
        finish();
        waleScalarProfile.workspaceBytes = arena.bytes - before;
    }
    // The face graph's per-face mixing record (allocated on first use of the
    // face graph: at install, on leaving the structured path, or by a host entry).
    void ensureGraphScalarWork() {
        if (!v.sgs || v.sc == 0 || v.sgsWork) return;
        const size_t before = arena.bytes;
        v.sgsWork = arena.get<double>(product(cfg.faces, 3));
        v.sgsCarrier = arena.get<int>(cfg.faces);
        waleScalarProfile.workspaceBytes += arena.bytes - before;
    }
    void uploadWaleScalarFields(const double* cellCp, const double* cellH, const double* fixedCp,
                                const double* fixedH) {
        require(!walePrInstalled, "Host WALE scalar upload cannot replace installed PR device properties");
        require(v.sgs, "WALE scalar closure is not selected");
        const bool uploadH = cellH || fixedH;
        if (v.pr > 0) {
            require(cellCp && (!cfg.fixed || fixedCp), "Missing WALE mixture heat capacities");
            require(firstFailure(cfg.cells, [&](size_t c) { return std::isfinite(cellCp[c]) && cellCp[c] > 0; })
                        == cfg.cells,
                    "Invalid WALE mixture heat capacity");
            require(firstFailure(cfg.fixed, [&](size_t c) { return std::isfinite(fixedCp[c]) && fixedCp[c] > 0; })
                        == cfg.fixed,
                    "Invalid fixed WALE mixture heat capacity");
        }
        if (v.sc > 0) {
            require(!uploadH || (cellH && (!cfg.fixed || fixedH)), "Incomplete WALE effective species enthalpies");
            if (uploadH) {
                const size_t n = cfg.cells * cfg.species, m = cfg.fixed * cfg.species;
                require(firstFailure(n, [&](size_t j) { return std::isfinite(cellH[j]); }) == n,
                        "Invalid WALE effective species enthalpy");
                require(firstFailure(m, [&](size_t j) { return std::isfinite(fixedH[j]); }) == m,
                        "Invalid fixed WALE effective species enthalpy");
            }
        }
        if (v.pr > 0) {
            upload(const_cast<double*>(v.mixCp), cellCp, cfg.cells);
            upload(const_cast<double*>(v.mixCp) + cfg.cells, fixedCp, cfg.fixed);
        }
        if (v.sc > 0 && uploadH) {
            packInto(const_cast<double*>(v.spH), cellH, cfg.cells, cfg.species, v.all, 0);
            packInto(const_cast<double*>(v.spH), fixedH, cfg.fixed, cfg.species, v.all, cfg.cells);
        }
        finish();
        scalarCp = v.pr == 0 || cellCp;
        scalarH = v.sc == 0 || uploadH;
        ++waleScalarProfile.fieldUploads;
        waleScalarProfile.fieldUploadBytes += (v.pr > 0 ? v.all * sizeof(double) : 0)
            + (v.sc > 0 && uploadH ? v.all * cfg.species * sizeof(double) : 0);
    }
    void uploadWaleScalarFieldsDevice(const double* cellCp, const double* cellH, const double* fixedCp,
                                      const double* fixedH, size_t cpStride, size_t hStride, cudaStream_t s) {
        require(!walePrInstalled, "Host WALE scalar upload cannot replace installed PR device properties");
        require(v.sgs, "WALE scalar closure is not selected");
        require(v.pr == 0 || cellCp, "Missing WALE mixture heat capacities");
        require((!cellCp || cpStride >= 1) && (!cellH || hStride >= cfg.species), "Invalid WALE scalar field strides");
        const double* cp = v.pr > 0 ? cellCp : nullptr;
        const double* h = v.sc > 0 ? cellH : nullptr;
        if (cp || h) {
            gatherScalarFields<<<gridFor(cfg.cells, 256), 256, 0, s>>>(cp, h, cpStride, hStride, cfg.cells, 0,
                                                                       cfg.species, v.all, const_cast<double*>(v.mixCp),
                                                                       const_cast<double*>(v.spH), flags);
            launched();
        }
        const double* fcp = v.pr > 0 ? fixedCp : nullptr;
        const double* fh = v.sc > 0 ? fixedH : nullptr;
        if (cfg.fixed && (fcp || fh)) {
            gatherScalarFields<<<gridFor(cfg.fixed, 256), 256, 0, s>>>(fcp, fh, cpStride, hStride, cfg.fixed,
                                                                       cfg.cells, cfg.species, v.all,
                                                                       const_cast<double*>(v.mixCp),
                                                                       const_cast<double*>(v.spH), flags);
            launched();
        }
        scalarCp = true;
        scalarH = v.sc == 0 || cellH || cfg.species == 1;
        ++waleScalarProfile.fieldUploads;
    }
    // Stage / CFL preconditions (src/reactiveTransport/reactiveTransport.cpp:1395-1397, 1415-1416).
    void requireCapillaryGeometry() const {
        require(!v.capillary || colorReady, "Capillary geometry must be uploaded for this stage");
    }
    void requireScalarFields(bool transport) const {
        if (!v.sgs) return;
        if (transport)
            require((v.pr == 0 || scalarCp) && (v.sc == 0 || scalarH),
                    "WALE scalar heat capacities/enthalpies were not uploaded for this thermodynamic stage");
        else
            require(v.pr == 0 || scalarCp, "WALE scalar heat capacities were not uploaded for this thermodynamic stage");
    }
    void uploadPrimitives(const ReactiveTransportPrimitive* primitive, const ReactiveTransportState* state) {
        require(primitive, "Null transport primitives");
        uploadState(state, primitive);
    }
};

}  // namespace
}  // namespace rb200

#include "transport_abi.inc"
