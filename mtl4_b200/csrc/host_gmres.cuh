// GMRES: filled in below the batch code; this stub keeps the ABI complete.
#pragma once
extern "C" int mtlg_gmres_impl(mtlg_ctx* c, mtlg_csr* A, mtlg_pc* L, mtlg_pc* R, mtlg_vec* x, const mtlg_vec* b,
                               const mtlg_iter_params* p, mtlg_iter_result* r)
{
    (void)c; (void)A; (void)L; (void)R; (void)x; (void)b; (void)p; (void)r;
    mtlg::set_error("GMRES not built yet");
    return MTLG_ERR_NOT_SUPPORTED;
}
