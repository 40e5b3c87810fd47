"""Empty stand-in: the registration path never plots."""
