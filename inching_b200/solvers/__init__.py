"""GPU eigensolvers for the ANM Hessian store."""
