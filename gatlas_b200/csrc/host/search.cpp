// Search-space enumeration; see search.hpp for the reference citations.
#include "search.hpp"

#include <cmath>

namespace gatlas {
namespace host {

std::vector<std::vector<size_t>> matmul_search(KernelMatmul &k, size_t vl, size_t maxBH, size_t maxWG, bool gemm,
                                               size_t M, size_t N, size_t K, bool tA, bool tB, long group,
                                               long bh, long xp) {
    std::vector<std::vector<size_t>> out;
    std::vector<size_t> a;
    auto push = [&]() {
        if (k.getParams(a)) {
            out.push_back(a);
            return true;
        }
        return false;
    };
    k.setGeneralizedMatmul(gemm);
    k.setMatrixDimensions(M, N, K);
    k.setDataLayout(tA, tB);
    if (group != -1) k.setWorkGroup((size_t)group);
    if (bh != -1) k.setInnerBlocking((size_t)bh, vl);
    if (xp != -1) k.setExtraParameter((size_t)xp);

    if (group != -1 && bh != -1 && xp != -1) {
        push();
    } else if (group != -1 && bh != -1) {
        for (size_t x = 0; x < k.totalVariations(); ++x) {
            k.setExtraParameter(x);
            push();
        }
    } else if (group != -1) {
        for (size_t h = vl; h <= maxBH; ++h) {
            k.setInnerBlocking(h, vl);
            for (size_t x = 0; x < k.totalVariations(); ++x) {
                k.setExtraParameter(x);
                push();
            }
        }
    } else {
        // largest valid square group down to 9, then 8 (the 64-thread wavefront of the 5870)
        const size_t largestPossible = (size_t)std::sqrt((double)kMaxWorkGroupSize);
        const size_t largest = maxWG < largestPossible ? maxWG : largestPossible;
        const size_t bhMin = bh != -1 ? (size_t)bh : vl, bhMax = bh != -1 ? (size_t)bh : maxBH;
        const size_t xMin = xp != -1 ? (size_t)xp : 0, xMax = xp != -1 ? (size_t)xp + 1 : k.totalVariations();
        for (size_t wg = largest; wg > 8; --wg) {
            k.setWorkGroup(wg);
            bool any = false;
            for (size_t h = bhMin; h <= bhMax; ++h) {
                k.setInnerBlocking(h, vl);
                for (size_t x = xMin; x < xMax; ++x) {
                    k.setExtraParameter(x);
                    if (push()) any = true;
                }
            }
            if (any) break;
        }
        k.setWorkGroup(8);
        for (size_t h = bhMin; h <= bhMax; ++h) {
            k.setInnerBlocking(h, vl);
            for (size_t x = xMin; x < xMax; ++x) {
                k.setExtraParameter(x);
                push();
            }
        }
    }
    return out;
}

std::vector<std::vector<size_t>> matvec_search(KernelMatvec &k, size_t vl, size_t maxBH, size_t maxWG, bool gemv,
                                               size_t M, size_t N, bool tA, long group, long bh, long xp) {
    std::vector<std::vector<size_t>> out;
    std::vector<size_t> a;
    auto push = [&]() {
        if (k.getParams(a)) {
            out.push_back(a);
            return true;
        }
        return false;
    };
    k.setGeneralizedMatvec(gemv);
    k.setMatrixDimensions(M, N);
    k.setDataLayout(tA);
    if (group != -1) k.setWorkGroup((size_t)group);
    if (bh != -1) k.setInnerBlocking((size_t)bh, vl);
    if (xp != -1) k.setExtraParameter((size_t)xp);

    if (group != -1 && bh != -1 && xp != -1) {
        push();
    } else if (group != -1 && bh != -1) {
        for (size_t x = 0; x < k.totalVariations(); ++x) {
            k.setExtraParameter(x);
            push();
        }
    } else if (group != -1) {
        for (size_t h = vl; h <= maxBH; ++h) {
            k.setInnerBlocking(h, vl);
            for (size_t x = 0; x < k.totalVariations(); ++x) {
                k.setExtraParameter(x);
                push();
            }
        }
    } else {
        const size_t largest = maxWG < kMaxWorkGroupSize ? maxWG : kMaxWorkGroupSize;
        const size_t bhMin = bh != -1 ? (size_t)bh : vl, bhMax = bh != -1 ? (size_t)bh : maxBH;
        const size_t xMin = xp != -1 ? (size_t)xp : 0, xMax = xp != -1 ? (size_t)xp + 1 : k.totalVariations();
        for (size_t wg = largest; wg > 64; --wg) {
            k.setWorkGroup(wg);
            bool any = false;
            for (size_t h = bhMin; h <= bhMax; ++h) {
                k.setInnerBlocking(h, vl);
                for (size_t x = xMin; x < xMax; ++x) {
                    k.setExtraParameter(x);
                    if (push()) any = true;
                }
            }
            if (any) break;
        }
        k.setWorkGroup(64);
        for (size_t h = bhMin; h <= bhMax; ++h) {
            k.setInnerBlocking(h, vl);
            for (size_t x = xMin; x < xMax; ++x) {
                k.setExtraParameter(x);
                push();
            }
        }
    }
    return out;
}

std::vector<std::vector<size_t>> saxpy_search(KernelSaxpy &k, size_t vl, size_t maxBH, size_t maxWG, size_t M,
                                              size_t N, long gh, long gw, long bh, long bw, long xp) {
    std::vector<std::vector<size_t>> out;
    std::vector<size_t> a;
    auto push = [&]() {
        if (k.getParams(a)) out.push_back(a);
    };
    k.setSaxpyDimensions(M, N);
    k.setVectorLength(vl);
    if (gh != -1) k.setWorkGroup((size_t)gh, gw == -1 ? 0 : (size_t)gw);
    if (bh != -1) k.setInnerBlocking((size_t)bh, bw == -1 ? 0 : (size_t)bw);
    if (xp != -1) k.setExtraParameter((size_t)xp);
    const size_t largest = maxWG < kMaxWorkGroupSize ? maxWG : kMaxWorkGroupSize;
    const bool oneD = (vl == N);

    if (gh != -1 && bh != -1 && xp != -1) {
        push();
    } else if (gh != -1 && bh == -1 && xp == -1) {
        if (oneD) {
            for (size_t h = 1; h <= maxBH; ++h) {
                k.setInnerBlocking(h, 0);
                for (size_t x = 0; x < k.totalVariations(); ++x) {
                    k.setExtraParameter(x);
                    push();
                }
            }
        } else {
            for (size_t h = 1; h <= maxBH; ++h)
                for (size_t w = 1; w <= 8; ++w) {
                    k.setInnerBlocking(h, w);
                    for (size_t x = 0; x < k.totalVariations(); ++x) {
                        k.setExtraParameter(x);
                        push();
                    }
                }
        }
    } else if (gh == -1 && bh != -1 && xp != -1) {
        if (oneD) {
            for (size_t wg = 64; wg <= largest; ++wg) {
                k.setWorkGroup(wg, 0);
                push();
            }
        } else {
            for (size_t h = 1; h <= largest; ++h)
                for (size_t w = 1; w <= largest; ++w)
                    if (h * w <= largest) {
                        k.setWorkGroup(h, w);
                        push();
                    }
        }
    } else {
        const size_t bhMin = bh != -1 ? (size_t)bh : 1, bhMax = bh != -1 ? (size_t)bh : maxBH;
        const size_t xMin = xp != -1 ? (size_t)xp : 0, xMax = xp != -1 ? (size_t)xp + 1 : k.totalVariations();
        if (oneD) {
            for (size_t wg = 64; wg <= largest; ++wg) {
                k.setWorkGroup(wg, 0);
                for (size_t h = bhMin; h <= bhMax; ++h) {
                    k.setInnerBlocking(h, 0);
                    for (size_t x = xMin; x < xMax; ++x) {
                        k.setExtraParameter(x);
                        push();
                    }
                }
            }
        } else {
            for (size_t wh = 1; wh <= largest; ++wh)
                for (size_t ww = 1; ww <= largest; ++ww)
                    if (wh * ww <= largest) {
                        k.setWorkGroup(wh, ww);
                        for (size_t h = bhMin; h <= bhMax; ++h)
                            for (size_t w = 1; w <= 8; ++w) {
                                k.setInnerBlocking(h, w);
                                for (size_t x = xMin; x < xMax; ++x) {
                                    k.setExtraParameter(x);
                                    push();
                                }
                            }
                    }
        }
    }
    return out;
}

}  // namespace host
}  // namespace gatlas
