//=============================================================================
// clg_ref_driver.cpp -- runs the reference's own CUDA implementation (CLGLib,
// built by oracle/ref/Makefile) on fields given as CLGBin files.
//
// Test infrastructure: its outputs pin the CPU oracle (tests/golden/ref_*.npz,
// written by tests/golden/make_ref_golden.py) and give the reference-GPU
// timings.  Nothing in the product links or runs it.
//
// Usage: clg_ref_driver <job.yaml>
//
// The YAML holds one block named Job, laid out as a test block of the
// reference's Bin/Debug/TestSuit_*.yaml files: an ordinary CLGLib parameter set (lattice, gauge read from an
// EFFT_CLGBinDouble file, one fermion field with FieldId 2, optional Solver /
// MSSolver blocks), initialised with appInitialCLG (Core/CLGLibManager.cpp:1149),
// plus a RefJob block read only by this driver:
//
//   RefJob:
//       SourceFile : in.bin            ## EFFT_CLGBin fermion source (FP64 build)
//       OutPrefix : out                ## outputs: <OutPrefix>.<op>.bin
//       Ops : [D, Ddagger, InverseD]   ## see below
//       ShiftRe : [2.0, 1.0]           ## complex shifts of the MultiShift ops
//       ShiftIm : [0.0, 0.0]
//       Repeat : 20                    ## applications timed by the Time* ops
//
// Ops: D, Ddagger, DD, DDdagger (CField::ApplyOperator, CField.h:203, on a copy
// of the source, in place as the reference does), InverseD, InverseDdagger,
// InverseDDdagger (the configured CSLASolver through ApplyOperator),
// MultiShiftD / MultiShiftDdagger / MultiShiftDDdagger (the configured
// CMultiShiftSolver::Solve, CMultiShiftSolver.h:38-47, x_n = (A + c_n)^-1 b),
// TimeD / TimeDdagger (Repeat applications in place, timed).  Every output is
// exported with CopyDataOutDouble (24 or 6 doubles per site, CLGBin order).
// One line "REFRESULT {json}" per op goes to stdout with the device time.
//=============================================================================
#include "CLGLib.h"
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

namespace {

struct DevTimer
{
    cudaEvent_t a, b;
    DevTimer() { cudaEventCreate(&a); cudaEventCreate(&b); }
    ~DevTimer() { cudaEventDestroy(a); cudaEventDestroy(b); }
    void start() { cudaDeviceSynchronize(); cudaEventRecord(a); }
    double stop_ms()
    {
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        return ms;
    }
};

bool write_field(const CField* f, const std::string& path)
{
    UINT size = 0;
    BYTE* bytes = f->CopyDataOutDouble(size);
    FILE* fp = fopen(path.c_str(), "wb");
    if (!fp) { free(bytes); return false; }
    const size_t n = fwrite(bytes, 1, size, fp);
    fclose(fp);
    free(bytes);
    return n == size;
}

bool op_of(const std::string& s, EFieldOperator& op)
{
    if (s == "D") op = EFO_F_D;
    else if (s == "Ddagger") op = EFO_F_Ddagger;
    else if (s == "DD") op = EFO_F_DD;
    else if (s == "DDdagger") op = EFO_F_DDdagger;
    else if (s == "InverseD") op = EFO_F_InverseD;
    else if (s == "InverseDdagger") op = EFO_F_InverseDdagger;
    else if (s == "InverseDDdagger") op = EFO_F_InverseDDdagger;
    else return false;
    return true;
}

}  // namespace

int main(int argc, char* argv[])
{
    if (argc < 2)
    {
        fprintf(stderr, "usage: %s job.yaml\n", argv[0]);
        return 2;
    }
    CParameters file;
    CYAMLParser::ParseFile(argv[1], file);
    CParameters params;
    if (!file.FetchParameterValue(_T("Job"), params))
    {
        fprintf(stderr, "no Job block in %s\n", argv[1]);
        return 2;
    }
    CParameters job;
    if (!params.FetchParameterValue(_T("RefJob"), job))
    {
        fprintf(stderr, "no RefJob block in %s\n", argv[1]);
        return 2;
    }
    CCString sSource, sPrefix;
    TArray<CCString> ops;
    if (!job.FetchStringValue(_T("SourceFile"), sSource) || !job.FetchStringValue(_T("OutPrefix"), sPrefix)
        || !job.FetchStringVectorValue(_T("Ops"), ops))
    {
        fprintf(stderr, "RefJob needs SourceFile, OutPrefix and Ops\n");
        return 2;
    }
    TArray<DOUBLE> shiftRe, shiftIm;
    job.FetchValueArrayDOUBLE(_T("ShiftRe"), shiftRe);
    job.FetchValueArrayDOUBLE(_T("ShiftIm"), shiftIm);
    INT iRepeat = 20;
    job.FetchValueINT(_T("Repeat"), iRepeat);

    if (!appInitialCLG(params))
    {
        fprintf(stderr, "appInitialCLG failed\n");
        return 3;
    }

    CFieldFermion* pSource = dynamic_cast<CFieldFermion*>(appGetLattice()->GetFieldById(2));
    if (NULL == pSource)
    {
        fprintf(stderr, "no fermion field with FieldId 2\n");
        appQuitCLG();
        return 3;
    }
    pSource->InitialFieldWithFile(sSource, EFFT_CLGBin);
    // the solvers' relative stopping rule reads the source's stored |b|^2
    // (set by InitialField for generated fields, not by a file load)
    pSource->m_fLength = pSource->Dot(pSource).x;
    checkCudaErrors(cudaDeviceSynchronize());

    const std::string prefix(sPrefix.c_str());
    DevTimer timer;
    int failures = 0;
    for (INT i = 0; i < ops.Num(); ++i)
    {
        const std::string name(ops[i].c_str());
        EFieldOperator op;
        if (name.rfind("MultiShift", 0) == 0)
        {
            if (!op_of(name.substr(10), op) || shiftRe.Num() == 0 || shiftRe.Num() != shiftIm.Num())
            {
                fprintf(stderr, "bad multi-shift op %s\n", name.c_str());
                ++failures;
                continue;
            }
            CMultiShiftSolver* pSolver = appGetMultiShiftSolver(2);
            if (NULL == pSolver)
            {
                fprintf(stderr, "no MSSolver configured\n");
                ++failures;
                continue;
            }
            TArray<CLGComplex> cn;
            TArray<CField*> xs;
            for (INT k = 0; k < shiftRe.Num(); ++k)
            {
                cn.AddItem(_make_cuComplex(static_cast<Real>(shiftRe[k]), static_cast<Real>(shiftIm[k])));
                xs.AddItem(pSource->GetCopy());
            }
            timer.start();
            const UBOOL ok = pSolver->Solve(xs, cn, pSource, _FIELDS, op);
            const double ms = timer.stop_ms();
            for (INT k = 0; k < xs.Num(); ++k)
            {
                char path[64];
                snprintf(path, sizeof(path), ".%s.%d.bin", name.c_str(), k);
                if (!write_field(xs[k], prefix + path)) ++failures;
                appSafeDelete(xs[k]);
            }
            printf("REFRESULT {\"op\": \"%s\", \"ok\": %d, \"ms\": %.6f, \"shifts\": %d}\n",
                name.c_str(), ok ? 1 : 0, ms, static_cast<int>(shiftRe.Num()));
        }
        else if (name.rfind("Time", 0) == 0)
        {
            if (!op_of(name.substr(4), op))
            {
                fprintf(stderr, "bad timed op %s\n", name.c_str());
                ++failures;
                continue;
            }
            CField* pWork = pSource->GetCopy();
            pWork->ApplyOperator(op, _FIELDS);  // untimed warm-up
            timer.start();
            for (INT r = 0; r < iRepeat; ++r)
            {
                pWork->ApplyOperator(op, _FIELDS);
            }
            const double ms = timer.stop_ms();
            printf("REFRESULT {\"op\": \"%s\", \"ok\": 1, \"ms\": %.6f, \"repeat\": %d, \"ms_per_apply\": %.6f}\n",
                name.c_str(), ms, iRepeat, ms / iRepeat);
            appSafeDelete(pWork);
        }
        else
        {
            if (!op_of(name, op))
            {
                fprintf(stderr, "unknown op %s\n", name.c_str());
                ++failures;
                continue;
            }
            CField* pWork = pSource->GetCopy();
            timer.start();
            const UBOOL ok = pWork->ApplyOperator(op, _FIELDS);
            const double ms = timer.stop_ms();
            if (!write_field(pWork, prefix + "." + name + ".bin")) ++failures;
            printf("REFRESULT {\"op\": \"%s\", \"ok\": %d, \"ms\": %.6f}\n", name.c_str(), ok ? 1 : 0, ms);
            appSafeDelete(pWork);
        }
        fflush(stdout);
    }
    // every output is written; the process ends here without the library's
    // teardown (appQuitCLG), which crashed on the host after the first job
    fflush(stdout);
    fflush(stderr);
    std::_Exit(failures == 0 ? 0 : 4);
}
