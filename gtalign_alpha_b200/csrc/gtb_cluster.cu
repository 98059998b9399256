// gtb_cluster.cu -- clustering of structures from their all-against-all
// records, as the reference's clustering writer does it (TdClustWriter.h,
// TdClustWriter.cpp): a distance per pair from the record, the progressive
// pointer representation (pi, lambda) of single linkage (SLINK, Sibson 1973)
// or complete linkage (CLINK, Defays 1977) over the structures in their
// order, clusters cut at the threshold, a representative per cluster.
//
// Host code only: the linkage is sequential over the structures (each new
// structure updates the pointer representation of all earlier ones) and
// takes O(n^2) time on the n^2 records the search has already produced.
#include <algorithm>
#include <cstring>
#include <vector>
#include "gtb200.h"

namespace {

constexpr float TOOBIG = 999.9f;   // lambda of a structure not yet merged (CLUST_TOOBIGDISTANCE)

// distance of structure q to an earlier structure i from the record of q
// (as query) against i (TdClustWriter.h:236-262); pairs the search did not
// align get the largest distance, as pairs the reference never compared do
float pair_distance(const float* rec, int lq, int li, const gtb_cluster_options& o) {
    const float big = o.measure == GTB_SORT_RMSD ? 100.0f : 1.0f;
    if (rec[GTB_OUT_ALNLENGTH] < 1.0f) return big;
    const float nalnres = (float)((int)rec[GTB_OUT_ALNLENGTH] - (int)rec[GTB_OUT_NGAPS]);
    const float tmq = rec[GTB_OUT_SCOREQ], tmr = rec[GTB_OUT_SCORER];
    const float grt = std::max(tmq, tmr);
    const float hmn = 0.0f < grt ? (2.f * tmq * tmr) / (tmq + tmr) : 0.0f;
    float d = std::max(0.0f, 1.0f - grt);
    if (o.measure == GTB_SORT_TMREF) d = std::max(0.0f, 1.0f - tmr);
    if (o.measure == GTB_SORT_TMQUERY) d = std::max(0.0f, 1.0f - tmq);
    if (o.measure == GTB_SORT_TMHARMONIC) d = std::max(0.0f, 1.0f - hmn);
    if (o.measure == GTB_SORT_RMSD) d = rec[GTB_OUT_RMSD];
    const float cov = o.coverage;
    const bool low = o.onesided ? (nalnres < cov * (float)li && nalnres < cov * (float)lq)
                                : (nalnres < cov * (float)li || nalnres < cov * (float)lq);
    return low ? big : d;
}

// SLINK step for structure n with distances mu[0..n-1] (TdClustWriter.h:408-430)
void slink(int n, std::vector<float>& mu, std::vector<int>& pi, std::vector<float>& lambda) {
    pi[n] = n;
    lambda[n] = TOOBIG;
    for (int i = 0; i < n; i++) {
        if (lambda[i] >= mu[i]) {
            mu[pi[i]] = std::min(mu[pi[i]], lambda[i]);
            lambda[i] = mu[i];
            pi[i] = n;
        }
        if (lambda[i] < mu[i]) mu[pi[i]] = std::min(mu[pi[i]], mu[i]);
    }
    for (int i = 0; i < n; i++)
        if (lambda[i] >= lambda[pi[i]]) pi[i] = n;
}

// CLINK step for structure n (TdClustWriter.h:438-488).  The reference keeps
// two of the relayed lambdas of step 7 in int variables, which drops their
// fractions; that is kept, so that the clusters are the reference's.
void clink(int n, std::vector<float>& mu, std::vector<int>& pi, std::vector<float>& lambda) {
    pi[n] = n;
    lambda[n] = TOOBIG;
    for (int i = 0; i < n; i++) {
        if (lambda[i] < mu[i]) {
            mu[pi[i]] = std::max(mu[pi[i]], mu[i]);
            mu[i] = TOOBIG;
        }
    }
    int a = n - 1;
    for (int k = 0; k < n; k++) {
        const int i = n - 1 - k;
        if (lambda[i] >= mu[pi[i]]) {
            if (mu[i] < mu[a]) a = i;
        }
        if (lambda[i] < mu[pi[i]]) mu[i] = TOOBIG;
    }
    int b = a, c = a;
    if (0 <= a) {
        b = pi[a]; pi[a] = n;
        c = (int)lambda[a]; lambda[a] = mu[a];
    }
    if (a < n - 1) {
        while (b < n - 1) {
            const int d = pi[b];
            pi[b] = n;
            const int e = (int)lambda[b];
            lambda[b] = (float)c;
            b = d;
            c = e;
        }
        if (b == n - 1) {
            pi[b] = n;
            lambda[b] = (float)c;
        }
    }
    for (int i = 0; i < n; i++)
        if (pi[pi[i]] == n && lambda[i] >= lambda[pi[i]]) pi[i] = n;
}

}  // namespace

struct gtb_clusterer {
    int n = 0, next = 0;
    gtb_cluster_options o{};
    std::vector<int> lens, pi;
    std::vector<float> lambda, mu;
};

static bool valid(const gtb_cluster_options& o) {
    return (o.linkage == GTB_LINKAGE_COMPLETE || o.linkage == GTB_LINKAGE_SINGLE) &&
           o.measure >= GTB_SORT_TMGREATER && o.measure <= GTB_SORT_RMSD &&
           (o.coverage > 0.0f && o.coverage <= 1.0f) && (o.threshold >= 0.0f && o.threshold < 100.0f);
}

extern "C" gtb_status gtb_cluster_create(int n, const int* lens, const gtb_cluster_options* opts,
                                         gtb_clusterer** out) {
    if (!out) return GTB_ERR_ARG;
    *out = nullptr;
    if (n < 1 || !lens || !opts || !valid(*opts)) return GTB_ERR_ARG;
    gtb_clusterer* c = new gtb_clusterer();
    c->n = n;
    c->o = *opts;
    c->lens.assign(lens, lens + n);
    c->pi.assign(n, 0);
    c->lambda.assign(n, 0.0f);
    c->mu.assign(n, 0.0f);
    *out = c;
    return GTB_OK;
}

// structure q's records against the structures before it, in order (the
// reference runs the linkage as each query's results arrive,
// TdClustWriter.cpp:229-249)
extern "C" gtb_status gtb_cluster_add(gtb_clusterer* c, int q, const float* rec) {
    if (!c || q != c->next || q >= c->n || (q > 0 && !rec)) return GTB_ERR_ARG;
    for (int i = 0; i < q; i++) c->mu[i] = pair_distance(rec + (long long)i * GTB_NOUT, c->lens[q], c->lens[i], c->o);
    if (c->o.linkage == GTB_LINKAGE_SINGLE) slink(q, c->mu, c->pi, c->lambda);
    else clink(q, c->mu, c->pi, c->lambda);
    c->next++;
    return GTB_OK;
}

extern "C" gtb_status gtb_cluster_finish(gtb_clusterer* cl, int* pi_out, float* lambda_out, int* member,
                                         int* offset, int* rep, int* ncl) {
    if (!cl || cl->next != cl->n || !member || !offset || !rep || !ncl) return GTB_ERR_ARG;
    const int n = cl->n;
    const gtb_cluster_options& o = cl->o;
    const std::vector<int>& pi = cl->pi;
    const std::vector<float>& lambda = cl->lambda;
    // clusters at the threshold (TdClustWriter.cpp:271-346): subclusters
    // ("layers") of structures, and clusters of subclusters
    const float thr = o.measure == GTB_SORT_RMSD ? o.threshold : std::max(0.0f, 1.0f - o.threshold);
    std::vector<std::vector<int>> inlayer, clusters;
    std::vector<int> tolayer(n, -1), toclusters;
    auto newcluster = [&](int a, int b) {
        const int lyr = (int)inlayer.size(), clt = (int)clusters.size();
        inlayer.push_back(b >= 0 ? std::vector<int>{a, b} : std::vector<int>{a});
        clusters.push_back(std::vector<int>{lyr});
        tolayer[a] = lyr;
        if (b >= 0) tolayer[b] = lyr;
        toclusters.resize(lyr + 1, -1);
        toclusters[lyr] = clt;
    };
    for (int q = 0; q < n; q++) {
        const int qq = pi[q];
        const int l1 = tolayer[q], l2 = tolayer[qq];
        if (lambda[q] <= thr) {
            if (l1 < 0 && l2 < 0) {
                newcluster(q, qq);
            } else if (0 <= l1 && 0 <= l2) {
                int c1 = toclusters[l1], c2 = toclusters[l2];
                if (clusters[c1].size() < clusters[c2].size()) std::swap(c1, c2);
                clusters[c1].insert(clusters[c1].end(), clusters[c2].begin(), clusters[c2].end());
                for (int l : clusters[c2]) toclusters[l] = c1;
                clusters[c2].clear();
            } else if (l1 < 0) {
                inlayer[l2].push_back(q);
                tolayer[q] = l2;
            } else {
                inlayer[l1].push_back(qq);
                tolayer[qq] = l1;
            }
        } else {
            if (l1 < 0) newcluster(q, -1);
            if (q != qq && l2 < 0) newcluster(qq, -1);
        }
    }

    // representatives (TdClustWriter.cpp:352-390): the member with the
    // smallest lambda; members listed representative first, then in the
    // order the writer prints them (TdClustWriter.cpp:505-545)
    int nc = 0, nm = 0;
    offset[0] = 0;
    for (const auto& cl : clusters) {
        int r = -1;
        float mind = TOOBIG;
        int sz = 0;
        for (int l : cl)
            for (int s : inlayer[l]) {
                if (lambda[s] < mind || r < 0) { mind = lambda[s]; r = s; }
                sz++;
            }
        if (sz == 0) continue;
        rep[nc] = r;
        member[nm++] = r;
        for (int l : cl)
            for (int s : inlayer[l])
                if (s != r) member[nm++] = s;
        offset[++nc] = nm;
    }
    *ncl = nc;
    if (pi_out) std::memcpy(pi_out, pi.data(), sizeof(int) * n);
    if (lambda_out) std::memcpy(lambda_out, lambda.data(), sizeof(float) * n);
    return GTB_OK;
}

extern "C" void gtb_cluster_destroy(gtb_clusterer* c) { delete c; }

extern "C" gtb_status gtb_cluster(int n, const float* alndata, const int* lens,
                                  const gtb_cluster_options* opts, int* pi_out, float* lambda_out,
                                  int* member, int* offset, int* rep, int* ncl) {
    if (n < 1 || !alndata) return GTB_ERR_ARG;
    gtb_clusterer* c = nullptr;
    gtb_status s = gtb_cluster_create(n, lens, opts, &c);
    for (int q = 0; s == GTB_OK && q < n; q++)
        s = gtb_cluster_add(c, q, alndata + (long long)q * n * GTB_NOUT);
    if (s == GTB_OK) s = gtb_cluster_finish(c, pi_out, lambda_out, member, offset, rep, ncl);
    gtb_cluster_destroy(c);
    return s;
}
