// ORACLE BUILD SHIM — test infrastructure, not product code.
//
// Declarations standing in for the ROOT classes the reference names (file IO
// of ROOT TTrees and the histograms of writeResult; src/Analysis.cu:27-31,
// 178-495, 1355-2512, include/Figure.cuh:7-11). ROOT is not installed on
// this machine or the GPU box. The reference's likelihood path (config.yml,
// .dat samples, getNLL, getHessian) does not touch ROOT; these stubs only let
// the sources compile unmodified: opening a ROOT file fails as a missing file
// does (TFile::Open returns null), and histogram or tree output does nothing.
#pragma once

#include <cstddef>

typedef long long Long64_t;
typedef int Int_t;
typedef double Double_t;

class TObject {
public:
    enum { kOverwrite = 2, kWriteDelete = 4 };
    virtual ~TObject() {}
    int Write(const char* = nullptr, int = 0, int = 0) const { return 0; }
};

class TDirectory : public TObject {
public:
    TDirectory* mkdir(const char*, const char* = "", bool = false) { return this; }
    TDirectory* GetDirectory(const char*, bool = false, const char* = "") { return this; }
    bool cd(const char* = nullptr) { return true; }
    TObject* Get(const char*) { return nullptr; }
    void Close(const char* = "") {}
};

class TFile : public TDirectory {
public:
    TFile() {}
    explicit TFile(const char*, const char* = "", const char* = "", int = 1) {}
    static TFile* Open(const char*, const char* = "", const char* = "", int = 1, int = 0) { return nullptr; }
    bool IsZombie() const { return true; }
    bool IsOpen() const { return false; }
};

class TTree : public TObject {
public:
    TTree() {}
    TTree(const char*, const char*, int = 99) {}
    template <class... A>
    TObject* Branch(A&&...) { return nullptr; }
    template <class... A>
    int SetBranchAddress(A&&...) { return 0; }
    long long GetEntries() const { return 0; }
    int GetEntry(long long = 0, int = 0) { return 0; }
    int Fill() { return 0; }
};

class TH1 : public TObject {
public:
    template <class... A>
    int Fill(A&&...) { return 0; }
    template <class... A>
    bool Add(A&&...) { return true; }
    template <class... A>
    void Scale(A&&...) {}
    template <class... A>
    void SetBins(A&&...) {}
    template <class... A>
    void SetBinContent(A&&...) {}
    template <class... A>
    double GetBinContent(A&&...) const { return 0.0; }
    void Reset(const char* = "") {}
    void Sumw2(bool = true) {}
    void SetDirectory(TDirectory*) {}
};

class TH1F : public TH1 {
public:
    template <class... A>
    explicit TH1F(A&&...) {}
};

class TH2F : public TH1 {
public:
    template <class... A>
    explicit TH2F(A&&...) {}
};

class TLorentzVector : public TObject {
public:
    double Px() const { return 0.0; }
    double Py() const { return 0.0; }
    double Pz() const { return 0.0; }
    double E() const { return 0.0; }
};

class TMatrixD : public TObject {
public:
    TMatrixD(int r, int c) : r_(r), c_(c), d_(new double[(size_t)(r > 0 ? r : 0) * (c > 0 ? c : 0) + 1]()) {}
    ~TMatrixD() { delete[] d_; }
    TMatrixD(const TMatrixD&) = delete;
    TMatrixD& operator=(const TMatrixD&) = delete;
    double& operator()(int i, int j) { return d_[(size_t)i * c_ + j]; }
    double operator()(int i, int j) const { return d_[(size_t)i * c_ + j]; }
    double* operator[](int i) { return d_ + (size_t)i * c_; }
    const double* operator[](int i) const { return d_ + (size_t)i * c_; }

private:
    int r_, c_;
    double* d_;
};

class TObjString : public TObject {
public:
    explicit TObjString(const char* = "") {}
};

class TROOT {
public:
    void SetBatch(bool = true) {}
};
inline TROOT* gROOT_stub() { static TROOT r; return &r; }
#define gROOT (gROOT_stub())
