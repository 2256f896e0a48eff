"""Drop-in projector modules mirroring ct_projector.projector.{cupy,numpy}."""
