// ref_harness.cu -- test driver around EZLDA's own sources (asherliu/LDA_SC20, EZLDA/).
//
// TEST INFRASTRUCTURE ONLY.  Built by oracle/ref/build_ref.py from the reference's
// unmodified .cu files (all but mainKernel.cu, whose main() this file replaces) plus
// legacy_shim.h, into oracle/_ref/ref_harness.  It calls the reference's host classes
// (Document, DTChunk, WTAll, WTD) and L2 wrappers in the order of EZLDA/mainKernel.cu and
// dumps their device state, so the oracle can be pinned to the reference's own outputs.
//
// Deviations from mainKernel.cu, all on the harness side:
//   - one CUDA stream (the reference's two streams only overlap chunks; each chunk still
//     uses its own per-stream buffers, streamId = chunk % numStreams);
//   - the curand states are allocated for (GridDim+3)*BlockDim threads and initialised
//     before the first sweep (EZLDA allocates GridDim*BlockDim although
//     UpdateProbKernelTrainD1 indexes up to 3*BlockDim past it, and never initialises
//     them for sweep 0, EZLDA/mainKernel.cu:103,164-168);
//   - SampleKernelD (LDAKernelTrainD, the kernel with the cross-CTA spin lock,
//     EZLDA/utility.cu:1613-1667) is never launched: the sweep and distribution modes
//     run corpora without dense words, where that kernel has no work.  Counts mode runs
//     only the rebuild and max-topic kernels, never a sampler.
//
// Modes:
//   counts <chunkdir> <outdir>            initial WT build + sweep-0 prologue + per-chunk
//                                         MaxTopicKernel/UpdateDTKernel; dumps all counts
//   sweeps <chunkdir> <outdir> <n>        n full sweeps; dumps the topics after each
//   dist   <chunkdir> <outdir> <reps> <stride>
//                                         reps independent sweeps from the initial topics;
//                                         histogram of the new topic of every stride-th token
//   time   <chunkdir> <outdir> <n>        n sweeps on EZLDA's two-stream schedule, timed
//                                         with its iterStart/iterStop events
//                                         (EZLDA/mainKernel.cu:158-347); writes per-sweep ms
#include "DTUpdateKernel.cuh"
#include "WTUpdateKernel.cuh"
#include "WTDenUpdateKernel.cuh"
#include "WTAddKernel.cuh"
#include "SamplingKernel.cuh"
#include "WTDense.cuh"
#include "Argument.cuh"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>
#include <vector>

using namespace std;

#define CK(x) do { cudaError_t e_ = (x); if (e_ != cudaSuccess) { fprintf(stderr, "%s:%d %s: %s\n", __FILE__, __LINE__, #x, cudaGetErrorString(e_)); exit(3); } } while (0)

struct Sizes {
    int maxTL, maxDT, maxWT, maxDoc, W, maxChunkWT, numD, numS, numChunks;
};

static Sizes read_sizes(const string& prefix) {
    Sizes s{};
    ifstream lv((prefix + "/lengthVec.txt").c_str());
    if (!(lv >> s.maxTL >> s.maxDT >> s.maxWT >> s.maxDoc >> s.W >> s.maxChunkWT >> s.numD >> s.numS)) {
        fprintf(stderr, "cannot read %s/lengthVec.txt\n", prefix.c_str());
        exit(2);
    }
    ifstream dl((prefix + "/docLength.txt").c_str());
    int v;
    s.numChunks = 0;
    while (dl >> v) s.numChunks++;
    if (s.numChunks <= 0 || s.numChunks % numStreams) {
        fprintf(stderr, "need an even, positive chunk count (have %d)\n", s.numChunks);
        exit(2);
    }
    return s;
}

template <class T>
static void dump_dev(const string& path, const T* dev, size_t n, cudaStream_t st) {
    vector<T> h(n);
    if (n) CK(cudaMemcpyAsync(h.data(), dev, n * sizeof(T), cudaMemcpyDeviceToHost, st));
    CK(cudaStreamSynchronize(st));
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    if (n) fwrite(h.data(), sizeof(T), n, f);
    fclose(f);
}

template <class T>
static void dump_host(const string& path, const T* h, size_t n) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    if (n) fwrite(h, sizeof(T), n, f);
    fclose(f);
}

struct Ref {
    Sizes s;
    string prefix;
    Document* doc = nullptr;
    DTChunk* dt = nullptr;
    WTD* wtd = nullptr;
    WTAll* wt = nullptr;
    cudaStream_t st;
    curandState* rs[numStreams];

    explicit Ref(const string& p) : prefix(p) {
        s = read_sizes(p);
        // EZLDA/mainKernel.cu:78-126
        doc = new Document(prefix, s.numChunks, s.maxTL, s.maxDoc, s.W);
        doc->loadDocument();
        doc->GPUMemAllocate();
        doc->deviceCounterMemAllocate();
        dt = new DTChunk(s.maxDT, s.maxDoc, s.numChunks);
        dt->loadDocDTLength(prefix);
        dt->CPUMemSet();
        dt->GPUMemAllocate();
        dt->loadDTCountOffset(prefix);
        wtd = new WTD(s.numD, s.W);
        wtd->GPUMemAllocate();
        wtd->GPUMemInit();
        CK(cudaStreamCreate(&st));
        for (int i = 0; i < numStreams; i++) CK(cudaMalloc(&rs[i], sizeof(curandState) * (GridDim + 3) * BlockDim));
        wt = new WTAll(s.maxWT, s.W, s.numChunks, s.maxChunkWT, s.numS);
        wt->CPUMemSet();
        wt->GPUMemAllocate();
        wt->GPUMemset(st);
        wt->loadWTLength(prefix);
        wt->loadWTCountOffset(prefix);
        wt->CPU2GPUCountOffset(st);
        init_rand();
        CK(cudaDeviceSynchronize());
    }

    void init_rand() {
        for (int i = 0; i < numStreams; i++) initRandState<<<GridDim + 3, BlockDim, 0, st>>>(rs[i]);
        CK(cudaGetLastError());
    }

    // EZLDA/mainKernel.cu:133-150: per-chunk dense WT histogram and chunk sparse WT.
    void initial_wt() {
        for (int c = 0; c < s.numChunks; c++) {
            const int sid = c % numStreams;
            doc->CPU2GPU(c, sid, st);
            wt->chunkCPU2GPUCountOffset(c, sid, st);
            wt->chunkGPUMemset(sid, st);
            UpdateWTDenKernel(*wtd, *wt, *doc, c, sid, st);
            UpdateWTKernel(*wt, *doc, c, sid, st);
            wt->chunkWTGPU2CPU(c, sid, st);
        }
        CK(cudaStreamSynchronize(st));
    }

    // EZLDA/mainKernel.cu:163-195: zero the global WT, n_k from the dense part, merge the
    // chunk sparse WTs into the global one.
    void prologue() {
        wt->GPUMemset(st);
        UpdateWTDenRowSumKernel(*wtd, *wt, st);
        for (int c = 0; c < s.numChunks; c++) {
            const int sid = c % numStreams;
            wt->chunkCPU2GPUCountOffset(c, sid, st);
            wt->chunkGPUMemset(sid, st);
            wt->chunkWTCPU2GPU(c, sid, st);
            WTAdditionKernel(*wt, *doc, sid, st);
        }
        doc->CPU2GPUPerplexity(st);
        CK(cudaStreamSynchronize(st));
    }

    // EZLDA/mainKernel.cu:211-228
    void chunk_stats(int c) {
        const int sid = c % numStreams;
        doc->CPU2GPU(c, sid, st);
        dt->GPUMemSet(c, sid, st);
        dt->CPU2GPUDTCountOffset(c, sid, st);
        MaxTopicKernel(*wt, *doc, *wtd, sid, st);
        UpdateDTKernel(*dt, *doc, sid, st);
        CK(cudaGetLastError());
    }

    // EZLDA/mainKernel.cu:245-279 (dense-word kernels skipped: no dense words)
    void chunk_sample(int c) {
        const int sid = c % numStreams;
        SampleKernel(*wt, *dt, *doc, rs[sid], sid, st);
        CK(cudaGetLastError());
    }

    // EZLDA/mainKernel.cu:298-304
    void chunk_wt(int c) {
        const int sid = c % numStreams;
        wt->chunkCPU2GPUCountOffset(c, sid, st);
        wt->chunkGPUMemset(sid, st);
        UpdateWTKernel(*wt, *doc, c, sid, st);
        wt->chunkWTGPU2CPU(c, sid, st);
        doc->GPU2CPU(c, sid, st);
    }

    // EZLDA/mainKernel.cu:355-359
    void epilogue() {
        wtd->GPUMemCopy(st);
        wtd->GPUMemset(st);
        for (int sid = 0; sid < numStreams; sid++) PerplexityKernel(*doc, sid, st);
        CK(cudaStreamSynchronize(st));
    }

    void sweep() {
        prologue();
        for (int c = 0; c < s.numChunks; c++) {
            chunk_stats(c);
            chunk_sample(c);
            chunk_wt(c);
        }
        epilogue();
    }

    size_t tokens() const {
        size_t n = 0;
        for (int c = 0; c < s.numChunks; c++) n += doc->TLLengthVec[c];
        return n;
    }

    vector<unsigned short> topics() const {
        vector<unsigned short> z;
        for (int c = 0; c < s.numChunks; c++)
            z.insert(z.end(), doc->docChunkVec[c].TLTopic, doc->docChunkVec[c].TLTopic + doc->TLLengthVec[c]);
        return z;
    }

    void set_topics(const vector<unsigned short>& z) {
        size_t o = 0;
        for (int c = 0; c < s.numChunks; c++) {
            memcpy(doc->docChunkVec[c].TLTopic, z.data() + o, sizeof(unsigned short) * doc->TLLengthVec[c]);
            o += doc->TLLengthVec[c];
        }
    }
};

// EZLDA/mainKernel.cu:158-347 with its two streams and events: prologue on stream 1,
// chunk c on stream c % 2 (the first chunk of stream 0 waits for the prologue), stream 1
// waits for stream 0's last chunk, iteration time between iterStart and iterStop.
static void mode_time(Ref& r, const string& out, int n) {
    if (r.s.numD != 0) { fprintf(stderr, "time mode needs a corpus without dense words\n"); exit(2); }
    cudaStream_t streams[numStreams];
    for (int i = 0; i < numStreams; i++) CK(cudaStreamCreateWithPriority(&streams[i], cudaStreamDefault, i));
    cudaEvent_t startEvent, iterStart, iterStop, stopEvents[numStreams];
    CK(cudaEventCreate(&startEvent));
    CK(cudaEventCreate(&iterStart));
    CK(cudaEventCreate(&iterStop));
    for (int i = 0; i < numStreams; i++) CK(cudaEventCreate(&stopEvents[i]));
    r.initial_wt();
    vector<float> ms(n);
    for (int it = 0; it < n; it++) {
        CK(cudaEventRecord(iterStart, streams[1]));
        r.wt->GPUMemset(streams[1]);
        if (it > 0)
            for (int sid = 0; sid < numStreams; sid++) initRandState<<<GridDim + 3, BlockDim, 0, streams[sid]>>>(r.rs[sid]);
        UpdateWTDenRowSumKernel(*r.wtd, *r.wt, streams[1]);
        for (int c = 0; c < r.s.numChunks; c++) {
            const int sid = c % numStreams;
            r.wt->chunkCPU2GPUCountOffset(c, sid, streams[1]);
            r.wt->chunkGPUMemset(sid, streams[1]);
            r.wt->chunkWTCPU2GPU(c, sid, streams[1]);
            WTAdditionKernel(*r.wt, *r.doc, sid, streams[1]);
        }
        r.doc->CPU2GPUPerplexity(streams[1]);
        CK(cudaEventRecord(startEvent, streams[1]));
        for (int c = 0; c < r.s.numChunks; c++) {
            const int sid = c % numStreams;
            cudaStream_t& st = streams[sid];
            r.doc->CPU2GPU(c, sid, st);
            r.dt->GPUMemSet(c, sid, st);
            r.dt->CPU2GPUDTCountOffset(c, sid, st);
            if (c < numStreams && sid != 1) CK(cudaStreamWaitEvent(st, startEvent, 0));
            MaxTopicKernel(*r.wt, *r.doc, *r.wtd, sid, st);
            UpdateDTKernel(*r.dt, *r.doc, sid, st);
            SampleKernel(*r.wt, *r.dt, *r.doc, r.rs[sid], sid, st);
            r.wt->chunkCPU2GPUCountOffset(c, sid, st);
            r.wt->chunkGPUMemset(sid, st);
            UpdateWTKernel(*r.wt, *r.doc, c, sid, st);
            r.wt->chunkWTGPU2CPU(c, sid, st);
            if (sid != 1) CK(cudaEventRecord(stopEvents[sid], st));
            r.doc->GPU2CPU(c, sid, st);
        }
        for (int sid = 0; sid < numStreams; sid++)
            if (sid != 1) CK(cudaStreamWaitEvent(streams[1], stopEvents[sid], 0));
        CK(cudaEventRecord(iterStop, streams[1]));
        CK(cudaEventSynchronize(iterStop));
        CK(cudaEventElapsedTime(&ms[it], iterStart, iterStop));
        r.wtd->GPUMemCopy(streams[1]);
        r.wtd->GPUMemset(streams[1]);
        CK(cudaStreamSynchronize(streams[1]));
    }
    dump_host(out + "/sweep_ms.f32", ms.data(), ms.size());
    vector<unsigned short> z = r.topics();
    dump_host(out + "/topics_last.u16", z.data(), z.size());
    printf("time ok: %d sweeps of %zu tokens\n", n, r.tokens());
}

static void mode_counts(Ref& r, const string& out) {
    r.initial_wt();
    r.prologue();
    dump_dev(out + "/nk.i32", r.wt->deviceWTRowSum, K, r.st);
    dump_dev(out + "/swt_nnz.i32", r.wt->deviceNZWTCount, r.s.numS, r.st);
    dump_dev(out + "/swt_idx.u16", r.wt->deviceWTIndex, r.s.maxWT, r.st);
    dump_dev(out + "/swt_val.u16", r.wt->deviceWTValue, r.s.maxWT, r.st);
    dump_dev(out + "/wt_off.i32", r.wt->deviceWTOffset, r.s.W, r.st);
    dump_dev(out + "/dwt.i32", r.wtd->deviceWTDense, (size_t)r.s.numD * K, r.st);
    for (int c = 0; c < r.s.numChunks; c++) {
        const int sid = c % numStreams;
        r.chunk_stats(c);
        const string p = out + "/c" + to_string(c) + "_";
        dump_dev(p + "meta.i64", r.doc->deviceMaxSecTopic[sid], r.doc->TLLengthVec[c], r.st);
        dump_dev(p + "dt_nnz.i32", r.dt->deviceNZDTCount[sid], r.dt->docLengthVec[c], r.st);
        dump_dev(p + "dt_ent.i32", r.dt->deviceDTIndexValue[sid], r.dt->DTLengthVec[c], r.st);
        dump_dev(p + "dt_off.i32", r.dt->deviceDTOffset[sid], r.dt->docLengthVec[c], r.st);
        if (c == 0) {
            dump_dev(out + "/wmax.u16", r.doc->deviceWordMaxTopic[sid], r.s.W, r.st);
            dump_dev(out + "/w2nd.u16", r.doc->deviceWordSecondMaxTopic[sid], r.s.W, r.st);
            dump_dev(out + "/w3rd.u16", r.doc->deviceWordThirdMaxTopic[sid], r.s.W, r.st);
            dump_dev(out + "/pmax.f32", r.doc->deviceWordMaxProb[sid], r.s.W, r.st);
            dump_dev(out + "/p2nd.f32", r.doc->deviceWordSecondMaxProb[sid], r.s.W, r.st);
            dump_dev(out + "/p3rd.f32", r.doc->deviceWordThirdMaxProb[sid], r.s.W, r.st);
            dump_dev(out + "/qarr.f32", r.doc->deviceQArray[sid], r.s.W, r.st);
        }
    }
    printf("counts ok: %d chunks, %zu tokens, %d dense words\n", r.s.numChunks, r.tokens(), r.s.numD);
}

static void mode_sweeps(Ref& r, const string& out, int n) {
    if (r.s.numD != 0) { fprintf(stderr, "sweeps mode needs a corpus without dense words\n"); exit(2); }
    r.initial_wt();
    for (int it = 0; it < n; it++) {
        if (it > 0) r.init_rand();  // EZLDA re-initialises the states every sweep (mainKernel.cu:164-168)
        r.sweep();
        vector<unsigned short> z = r.topics();
        dump_host(out + "/topics_" + to_string(it) + ".u16", z.data(), z.size());
    }
    printf("sweeps ok: %d sweeps of %zu tokens\n", n, r.tokens());
}

static void mode_dist(Ref& r, const string& out, int reps, int stride) {
    if (r.s.numD != 0) { fprintf(stderr, "dist mode needs a corpus without dense words\n"); exit(2); }
    const vector<unsigned short> z0 = r.topics();
    vector<long long> tracked;
    for (size_t i = 0; i < z0.size(); i += stride) tracked.push_back((long long)i);
    vector<int> hist(tracked.size() * K, 0);
    for (int rep = 0; rep < reps; rep++) {
        r.set_topics(z0);
        r.initial_wt();
        r.init_rand();
        r.sweep();
        vector<unsigned short> z = r.topics();
        for (size_t t = 0; t < tracked.size(); t++) {
            const int k = z[tracked[t]];
            if (k >= 1 && k <= K) hist[t * K + (k - 1)]++;
        }
    }
    dump_host(out + "/dist_tracked.i64", tracked.data(), tracked.size());
    dump_host(out + "/dist_hist.i32", hist.data(), hist.size());
    printf("dist ok: %d reps, %zu tracked tokens\n", reps, tracked.size());
}

int main(int argc, char** argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: %s counts|sweeps|dist <chunkdir> <outdir> [n|reps stride]\n", argv[0]);
        return 2;
    }
    const string mode = argv[1], dir = argv[2], out = argv[3];
    Ref r(dir);
    if (mode == "counts") mode_counts(r, out);
    else if (mode == "sweeps" && argc >= 5) mode_sweeps(r, out, atoi(argv[4]));
    else if (mode == "dist" && argc >= 6) mode_dist(r, out, atoi(argv[4]), atoi(argv[5]));
    else if (mode == "time" && argc >= 5) mode_time(r, out, atoi(argv[4]));
    else { fprintf(stderr, "bad mode\n"); return 2; }
    CK(cudaDeviceSynchronize());
    return 0;
}
